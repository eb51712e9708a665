// bulk_bw.cu -- per-SM throughput of TMA bulk copies (cp.async.bulk, global
// -> shared, no multicast) as the EVP tile kernel uses them: a producer warp
// fills an S-stage shared-memory ring with tiles of `ncopies` field copies of
// `copy_bytes` each, read from field-major arrays larger than L2; a consumer
// warp releases each stage as soon as it lands.  Reports GB/s over the whole
// GPU for several (copies, copy size, stages) shapes.  Every mbarrier wait is
// bounded (1 s, %globaltimer) and reports a timeout instead of hanging.
//   make -C cice-evp1d_b200 diag && cice-evp1d_b200/diag/bulk_bw
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

namespace {

constexpr unsigned long long kWaitNs = 1000000000ull;

__device__ __forceinline__ uint32_t sa(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long gns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool try_wait(unsigned long long *b, uint32_t par) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(sa(b)), "r"(par)
      : "memory");
  return ok != 0;
}
__device__ bool wait(unsigned long long *b, uint32_t par, int *err) {
  const unsigned long long t0 = gns();
  while (!try_wait(b, par))
    if (gns() - t0 > kWaitNs) {
      atomicExch(err, 1);
      return false;
    }
  return true;
}

__global__ void k_bulk(const char *src, size_t field_stride, int ntiles, int nt_field,
                       int ncopies, int copy_bytes, int stages, int *err) {
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned long long *full = reinterpret_cast<unsigned long long *>(sm);
  unsigned long long *empty = full + 8;
  unsigned char *buf = sm + 128;
  const int tile_bytes = ncopies * copy_bytes;
  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sa(&full[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sa(&empty[s])));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  int n = 0;
  if (threadIdx.x < 32) {  // producer
    bool ok = true;
    for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, n++) {
      const int s = n % stages;
      const uint32_t use = (uint32_t)(n / stages);
      int w = 1;
      if (n >= stages && lane == 0) w = wait(&empty[s], (use - 1) & 1, err) ? 1 : 0;
      w = __shfl_sync(0xffffffffu, w, 0);
      if (!w) {
        ok = false;
        break;
      }
      if (lane == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa(&full[s])),
                     "r"(tile_bytes)
                     : "memory");
      __syncwarp();
      for (int k = lane; k < ncopies; k += 32) {
        const char *g = src + (size_t)k * field_stride + (size_t)(t % nt_field) * copy_bytes;
        unsigned char *d = buf + (size_t)s * tile_bytes + (size_t)k * copy_bytes;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
                "r"(sa(d)),
            "l"(g), "r"(copy_bytes), "r"(sa(&full[s]))
            : "memory");
      }
    }
    // drain: every issued stage must land before exit
    if (lane == 0)
      for (int k = n - stages; k < n; k++)
        if (k >= 0) wait(&full[k % stages], (uint32_t)(k / stages) & 1, err);
  } else if (threadIdx.x < 64) {  // consumer
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, n++) {
      const int s = n % stages;
      if (lane == 0) {
        if (!wait(&full[s], (uint32_t)(n / stages) & 1, err)) break;
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sa(&empty[s])) : "memory");
      }
      __syncwarp();
    }
  }
}

}  // namespace

int main() {
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  const size_t total = (size_t)4 << 30;  // 4 GiB of source, well above L2
  char *src = nullptr;
  int *err = nullptr;
  if (cudaMalloc(&src, total) != cudaSuccess || cudaMalloc(&err, 4) != cudaSuccess) {
    printf("allocation failed\n");
    return 1;
  }
  cudaMemset(src, 1, total);
  cudaMemset(err, 0, 4);
  struct Shape {
    int ncopies, copy_bytes, stages;
  };
  const Shape shapes[] = {
      {36, 2048, 1}, {36, 2048, 2}, {36, 2048, 3},    // the EVP tile: 36 fields x 256 doubles
      {1, 73728, 2}, {4, 18432, 2}, {9, 8192, 2},      // the same bytes in fewer copies
      {18, 2048, 2}, {18, 2048, 4}, {18, 2048, 6},     // half tiles, more stages
      {36, 1024, 2}, {36, 1024, 4}, {36, 1024, 5},     // 128-point tiles
      {36, 2048, -1}, {36, 2048, -2}, {1, 73728, -1},  // from L2
      {1, 73728, 1}, {2, 36864, 1}, {4, 18432, 1},      // one tile in flight, fewer copies
      {15, 4096, 1}, {9, 8192, 1},
  };
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  printf("copies x bytes, stages, tile KB, GB/s (whole GPU), per SM GB/s\n");
  for (const Shape &sh : shapes) {
    // field arrays start on 256-byte boundaries (bulk copies need 16); a
    // negative stage count reads a 24 MB window again and again (L2 hits)
    const bool l2 = sh.stages < 0;
    const int stages = l2 ? -sh.stages : sh.stages;
    const size_t span = l2 ? ((size_t)24 << 20) : total;
    const size_t field_stride = (span / (size_t)sh.ncopies) & ~(size_t)255;
    const int nt_field = (int)(field_stride / (size_t)sh.copy_bytes);
    const int ntiles = l2 ? nt_field * 64 : nt_field;
    const int smem = 128 + stages * sh.ncopies * sh.copy_bytes;
    if (cudaFuncSetAttribute(k_bulk, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess) {
      printf("%d x %d, %d stages: shared memory %d not available\n", sh.ncopies, sh.copy_bytes,
             stages, smem);
      continue;
    }
    for (int rep = 0; rep < 2; rep++) {
      cudaEventRecord(e0);
      k_bulk<<<sms, 64, smem>>>(src, field_stride, ntiles, nt_field, sh.ncopies, sh.copy_bytes,
                                stages, err);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    int herr = 0;
    cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
    const cudaError_t ce = cudaGetLastError();
    const double bytes = (double)ntiles * sh.ncopies * sh.copy_bytes;
    printf("%2d x %6d, %d stages%s, %6.1f KB: %7.0f GB/s  %5.1f per SM%s%s\n", sh.ncopies,
           sh.copy_bytes, stages, l2 ? " (L2)" : "", sh.ncopies * sh.copy_bytes / 1024.0, bytes / ms / 1e6,
           bytes / ms / 1e6 / sms, herr ? "  (a wait timed out)" : "",
           ce != cudaSuccess ? cudaGetErrorString(ce) : "");
    if (herr || ce != cudaSuccess) break;
  }
  cudaFree(src);
  cudaFree(err);
  return 0;
}
