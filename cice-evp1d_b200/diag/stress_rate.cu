// stress_rate.cu -- throughput of the per-point EVP stress code against the
// number of warps per SM.  One block per SM; every thread runs the library's
// strain_rates + stress_update (csrc/evp_math.cuh, -fmad=false) on inputs in
// shared memory, writes its 8 str values to shared memory and its 12 new
// stresses to global memory, with one block barrier per round, as a tile of
// the TMA kernel does.  Reports points per microsecond per SM.
//   make -C cice-evp1d_b200 diag && cice-evp1d_b200/diag/stress_rate
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "evp_math.cuh"
using namespace evp;
constexpr int NP = 256;
template <int W>
__global__ void __launch_bounds__(W * 32, 1) k(Params p, int rounds, double *gout, double *sink) {
  extern __shared__ double sm[];
  double (*f)[NP] = reinterpret_cast<double (*)[NP]>(sm);
  double *u = sm + 19 * NP, *v = u + NP + 128;
  double (*str)[W * 32] = reinterpret_cast<double (*)[W * 32]>(v + NP + 128);
  uint32_t *lc = reinterpret_cast<uint32_t *>(&str[8][0]);
  const int tid = threadIdx.x;
  for (int i = tid; i < NP; i += blockDim.x) {
    f[0][i] = 1e4 + i; f[1][i] = 1.1e4 + i; f[2][i] = 1e4 + 3 * i; f[3][i] = 1e4 + 2 * i;
    f[4][i] = 1e4 + 5 * i; f[5][i] = 1e4 + 7 * i; f[6][i] = 2e4 + i;
    for (int k2 = 0; k2 < 12; k2++) f[7 + k2][i] = 1e3 * (k2 + 1) + i;
    lc[i] = (uint32_t)(((i + 1) % 384) | (((i + 17) % 384) << 10) | (((i + 33) % 384) << 20));
  }
  for (int i = tid; i < NP + 128; i += blockDim.x) { u[i] = 1e-3 * (i % 37); v[i] = -1e-3 * (i % 29); }
  __syncthreads();
  const int c = tid % NP;
  double acc = 0;
  for (int r = 0; r < rounds; r++) {
    const uint32_t l = lc[c];
    const int iee = l & 1023, ine = (l >> 10) & 1023, ise = (l >> 20) & 1023;
    Corners cr;
    cr.ucc = u[c]; cr.vcc = v[c]; cr.uee = u[iee]; cr.vee = v[iee];
    cr.une = u[ine]; cr.vne = v[ine]; cr.use = u[ise]; cr.vse = v[ise];
    const Geom gm = make_geom(f[0][c], f[1][c], f[2][c], f[3][c], f[4][c], f[5][c], p.deltaminEVP);
    const Strain sr = strain_rates(cr, gm, p.e_factor);
    double s12[12], out[8];
#pragma unroll
    for (int k2 = 0; k2 < 12; k2++) s12[k2] = f[7 + k2][c] + r;
    stress_update(s12, out, sr, f[6][c], gm, p);
#pragma unroll
    for (int k2 = 0; k2 < 12; k2++) gout[(size_t)k2 * 148 * 1024 + blockIdx.x * 1024 + tid] = s12[k2];
#pragma unroll
    for (int k2 = 0; k2 < 8; k2++) str[k2][tid] = out[k2];
    __syncthreads();
    acc += str[(r & 7)][(tid + 1) % blockDim.x];
  }
  if (acc == 1.2345) sink[0] = acc;
}
template <int W> void run(Params p, double *g, double *s, int sms) {
  cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
  const int rounds = 2000;
  for (int rep = 0; rep < 2; rep++) {
    cudaEventRecord(e0);
    const int smem = (19 * NP + 2 * (NP + 128) + 8 * W * 32) * 8 + NP * 4;
    cudaFuncSetAttribute(k<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k<W><<<sms, W * 32, smem>>>(p, rounds, g, s);
    cudaEventRecord(e1); cudaEventSynchronize(e1);
    float ms; cudaEventElapsedTime(&ms, e0, e1);
    cudaFuncAttributes at; cudaFuncGetAttributes(&at, k<W>);
    if (rep) printf("%2d warps/SM (%3d regs): %.3f ns per round, %.1f points per us per SM  %s\n", W, at.numRegs,
                    1e6 * ms / rounds, W * 32.0 * rounds / (ms * 1e3), cudaGetErrorString(cudaGetLastError()));
  }
}
int main() {
  int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  double *g, *s; cudaMalloc(&g, sizeof(double) * 12 * 148 * 1024); cudaMalloc(&s, 8);
  Params p{};
  p.arlx1i = 1.0 / 300; p.denom1 = 1.0 / (1 + p.arlx1i); p.brlx = 300; p.capping = 1; p.e_factor = 0.25;
  p.epp2i = 0.25; p.deltaminEVP = 2e-9; p.revp = 0; p.Ktens = 0; p.u0 = 5e-5; p.cosw = 1; p.sinw = 0; p.rhow = 1026;
  run<8>(p, g, s, sms); run<10>(p, g, s, sms); run<12>(p, g, s, sms); run<16>(p, g, s, sms);
  run<20>(p, g, s, sms); run<24>(p, g, s, sms);
  return 0;
}
