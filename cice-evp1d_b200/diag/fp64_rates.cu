// fp64_rates.cu -- FP64 throughput of add, mul+add, IEEE division and square
// root on one GPU (one block per SM, 4..32 warps per SM, each thread running
// 8 independent chains).  The EVP kernels must use CUDA's correctly rounded
// FP64 division and sqrt; their rate bounds the solver's arithmetic.
//   make -C cice-evp1d_b200 diag && cice-evp1d_b200/diag/fp64_rates
#include <cstdio>
#include <cuda_runtime.h>
template <int OP>
__global__ void k(double *out, int iters, double s) {
  double x[8];
  for (int i = 0; i < 8; i++) x[i] = 1.0 + 1e-3 * (threadIdx.x + i);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      if (OP == 0) x[i] = x[i] * s + 1e-9;          // mul+add (2 ops)
      if (OP == 1) x[i] = s / x[i] + 0.5;           // div (+add)
      if (OP == 2) x[i] = sqrt(x[i]) + 0.5;         // sqrt (+add)
      if (OP == 3) x[i] = x[i] + s;                 // add
    }
  }
  double r = 0; for (int i = 0; i < 8; i++) r += x[i];
  if (r == 12345.678) out[0] = r;
}
int main() {
  double *o; cudaMalloc(&o, 8);
  int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  const char *names[4] = {"mul+add", "div+add", "sqrt+add", "add"};
  for (int op = 0; op < 4; op++) for (int warps = 4; warps <= 32; warps *= 2) {
    int iters = op == 1 || op == 2 ? 200 : 2000;
    dim3 g(sms), b(32 * warps);
    cudaEvent_t a, c; cudaEventCreate(&a); cudaEventCreate(&c);
    auto launch = [&]() {
      if (op == 0) k<0><<<g, b>>>(o, iters, 1.0000001);
      if (op == 1) k<1><<<g, b>>>(o, iters, 1.0000001);
      if (op == 2) k<2><<<g, b>>>(o, iters, 1.0000001);
      if (op == 3) k<3><<<g, b>>>(o, iters, 1.0000001);
    };
    launch(); cudaDeviceSynchronize();
    cudaEventRecord(a); for (int r = 0; r < 5; r++) launch(); cudaEventRecord(c); cudaEventSynchronize(c);
    float ms; cudaEventElapsedTime(&ms, a, c); ms /= 5;
    double ops = (double)sms * b.x * iters * 8;
    int clk; cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, 0);
    double cyc = ms * 1e-3 * clk * 1e3;
    printf("%-9s warps/SM=%2d  %.3f ms  %.2f Gop/s  %.2f op/cycle/SM\n", names[op], warps, ms, ops / ms / 1e6, ops / cyc / sms);
  }
  return 0;
}
