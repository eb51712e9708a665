// evp_kernels_tma.cu -- the fused EVP subcycle as a persistent, TMA-fed
// producer/consumer kernel (sm_100a).
//
// One CTA per SM walks the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...
// A producer warp stages each tile into a two-slot shared-memory ring:
//   - the tile's owned points are contiguous slots, so each per-point field
//     (7 stress inputs, 12 stresses, 13 stepu inputs, u, v and two packed
//     index words) arrives with one cp.async.bulk (TMA) copy, completing on
//     the stage's mbarrier with complete_tx;
//   - the forward-halo points (recomputed stress) and the extra velocity
//     points of the stencil are gathered with 4/8-byte cp.async, whose
//     completion arrives on the same mbarrier (cp.async.mbarrier.arrive).
// Ten consumer warps (one thread per compute-set point: 256 owned + 64 halo)
// compute stress from shared memory into the shared str table, then stepu
// for the owned points, writing the new stresses and velocities to the other
// ping-pong buffer.  While they compute tile k the producer loads tile k+1.
//
// Every mbarrier wait is bounded by %globaltimer (kWaitNs): on expiry the
// kernel records an error code, every thread of the consumer group leaves the
// tile loop together, and the producer waits (bounded) for the copies it has
// issued before it exits, so nothing is left in flight.
#include <cstdint>

#include "evp_kernels.cuh"
#include "evp_tiles.h"

namespace evp {

namespace {

constexpr int kStages = 2;
constexpr int kConsumers = kTileOwned + kTileHalo;  // 320 = 10 warps
constexpr int kThreads = kConsumers + 32;           // + 1 producer warp
constexpr int kUV = kTileOwned + kTileUvx;
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s

struct Stage {
  double sf[kTmaStressFields][kTileOwned];  // dxT..HTNm1, strength, 12 stresses
  double uf[kTmaStepuFields][kTileOwned];   // stepu inputs
  double u[kUV];
  double v[kUV];
  uint32_t meta[kTileOwned];
  uint32_t lcor[kTileOwned];
  double hf[kTmaStressFields][kTileHalo];
  uint32_t hmeta[kTileHalo];
  uint32_t hlcc[kTileHalo];
  uint32_t hlcor[kTileHalo];
};

struct Smem {
  Stage st[kStages];
  double str[8][kZeroSlot + 1];
  unsigned long long full[kStages];
  unsigned long long empty[kStages];
  int abort_flag;
};

static_assert(sizeof(Stage) % 16 == 0, "stage must keep 16-byte alignment");

// ---------------- PTX helpers -------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase of parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity,
                                          int *err, int code) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > kWaitNs) {
      atomicMax(err, code);
      return false;
    }
  }
  return true;
}

// TMA bulk copy global -> shared, completing `bytes` on `bar` (no multicast).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}

__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}

// The barrier's pending count drops by one once this thread's earlier
// cp.async copies have landed.
__device__ __forceinline__ void cp_async_arrive(unsigned long long *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void consumer_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"(kConsumers) : "memory");
}

// ---------------- the kernel ---------------------------------------------------
template <bool kLast>
__global__ void __launch_bounds__(kThreads, 1) k_tma(TmaArgs a, Params p) {
  extern __shared__ unsigned char smem_raw[];
  Smem &S = *reinterpret_cast<Smem *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&S.full[s], 1 + 32);  // expect_tx arrival + 32 cp.async lanes
      mbar_init(&S.empty[s], 1);      // one consumer arrival per use
    }
    S.abort_flag = 0;
    mbar_fence_init();
  }
  if (tid < 8) S.str[tid][kZeroSlot] = 0.0;
  __syncthreads();

  if (tid >= kConsumers) {
    // ======================= producer warp ==============================
    const int lane = tid - kConsumers;
    int issued = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
      const int s = issued % kStages;
      const uint32_t use = (uint32_t)(issued / kStages);
      if (issued >= kStages) {
        int w = 1;
        if (lane == 0) w = mbar_wait(&S.empty[s], (use - 1) & 1, a.err, 2) ? 1 : 0;
        w = __shfl_sync(0xffffffffu, w, 0);
        if (!w) {
          ok = false;
          break;
        }
      }
      Stage &st = S.st[s];
      const int off = a.tile_off[t], cnt = a.tile_cnt[t];
      const uint32_t n4 = (uint32_t)((cnt + 3) & ~3);
      if (lane == 0) {
        const uint32_t b8 = n4 * 8u, b4 = n4 * 4u;
        mbar_arrive_expect_tx(&S.full[s],
                              (kTmaStressFields + kTmaStepuFields + 2) * b8 + 2 * b4);
        for (int f = 0; f < kTmaStressFields; f++) bulk_g2s(st.sf[f], a.sf[f] + off, b8, &S.full[s]);
        for (int f = 0; f < kTmaStepuFields; f++) bulk_g2s(st.uf[f], a.uf[f] + off, b8, &S.full[s]);
        bulk_g2s(st.u, a.u_in + off, b8, &S.full[s]);
        bulk_g2s(st.v, a.v_in + off, b8, &S.full[s]);
        bulk_g2s(st.meta, a.meta + off, b4, &S.full[s]);
        bulk_g2s(st.lcor, a.lcor + off, b4, &S.full[s]);
      }
      const int xo = a.uvx_off[t], nx = a.uvx_cnt[t];
      for (int x = lane; x < nx; x += 32) {
        const int g = a.uvx_idx[xo + x];
        cp_async8(&st.u[kTileOwned + x], a.u_in + g);
        cp_async8(&st.v[kTileOwned + x], a.v_in + g);
      }
      const int ho = a.halo_off[t], nh = a.halo_cnt[t];
      for (int h = lane; h < nh; h += 32) {
        const int g = a.halo_idx[ho + h];
        for (int f = 0; f < kTmaStressFields; f++) cp_async8(&st.hf[f][h], a.sf[f] + g);
        cp_async4(&st.hmeta[h], a.meta + g);
        cp_async4(&st.hlcc[h], a.halo_lcc + ho + h);
        cp_async4(&st.hlcor[h], a.halo_lcor + ho + h);
      }
      cp_async_arrive(&S.full[s]);
      issued++;
    }
    if (!ok) {
      // Consumers stopped early: wait (bounded) until every issued stage has
      // landed so that no copy targets shared memory after the CTA exits.
      for (int k = issued - kStages; k < issued; k++) {
        if (k < 0) continue;
        if (lane == 0) mbar_wait(&S.full[k % kStages], (uint32_t)(k / kStages) & 1, a.err, 3);
      }
      __syncwarp();
    }
    return;
  }

  // ========================= consumers ===================================
  const int c = tid;  // compute-set index: owned c < 256, halo 256 + h
  int it = 0;
  for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, it++) {
    const int s = it % kStages;
    const uint32_t use = (uint32_t)(it / kStages);
    if (!mbar_wait(&S.full[s], use & 1, a.err, 1)) S.abort_flag = 1;
    consumer_sync();
    if (S.abort_flag) break;
    const Stage &st = S.st[s];
    const int off = a.tile_off[t], cnt = a.tile_cnt[t], nh = a.halo_cnt[t];

    // ---------------- phase 1: stress ------------------------------------
    const bool own = c < kTileOwned;
    const int h = c - kTileOwned;
    if (own ? c < cnt : h < nh) {
      const uint32_t m = own ? st.meta[c] : st.hmeta[h];
      double out[8];
      if ((m >> 30) & kSkipT) {
#pragma unroll
        for (int k = 0; k < 8; k++) out[k] = 0.0;
      } else {
        const double *F = own ? &st.sf[0][c] : &st.hf[0][h];
        const int fs = own ? kTileOwned : kTileHalo;
        const uint32_t lc = own ? st.lcor[c] : st.hlcor[h];
        const int cc = own ? c : (int)st.hlcc[h];
        const int iee = lc & kLnbMask, ine = (lc >> kLnbBits) & kLnbMask;
        const int ise = (lc >> (2 * kLnbBits)) & kLnbMask;
        Corners cr;
        cr.ucc = st.u[cc];
        cr.vcc = st.v[cc];
        cr.uee = st.u[iee];
        cr.vee = st.v[iee];
        cr.une = st.u[ine];
        cr.vne = st.v[ine];
        cr.use = st.u[ise];
        cr.vse = st.v[ise];
        const Geom gm = make_geom(F[0 * fs], F[1 * fs], F[2 * fs], F[3 * fs], F[4 * fs],
                                  F[5 * fs], p.deltaminEVP);
        const Strain sr = strain_rates(cr, gm, p.e_factor);
        double s12[12];
#pragma unroll
        for (int k = 0; k < 12; k++) s12[k] = F[(7 + k) * fs];
        stress_update(s12, out, sr, F[6 * fs], gm, p);
        if (own) {
#pragma unroll
          for (int k = 0; k < 12; k++) a.s_out[k][off + c] = s12[k];
        }
      }
#pragma unroll
      for (int k = 0; k < 8; k++) S.str[k][c] = out[k];
      if (kLast && own) {
#pragma unroll
        for (int k = 0; k < 8; k++) a.str_out[k][off + c] = out[k];
      }
    }
    consumer_sync();

    // ---------------- phase 2: stepu on owned points ------------------------
    if (c < cnt) {
      const uint32_t m = st.meta[c];
      if (!((m >> 30) & kSkipU)) {
        const int lnw = m & kLnbMask, lsw = (m >> kLnbBits) & kLnbMask;
        const int lsse = (m >> (2 * kLnbBits)) & kLnbMask;
        StepuIn in;
        in.uold = st.u[c];
        in.vold = st.v[c];
        in.kvrel = st.uf[0][c];
        in.uocn = st.uf[1][c];
        in.vocn = st.uf[2][c];
        in.waterx = st.uf[3][c];
        in.watery = st.uf[4][c];
        in.forcex = st.uf[5][c];
        in.forcey = st.uf[6][c];
        in.umassdti = st.uf[7][c];
        in.fm = st.uf[8][c];
        in.uarear = st.uf[9][c];
        in.Tbu = st.uf[10][c];
        in.uinit = st.uf[11][c];
        in.vinit = st.uf[12][c];
        in.s1 = S.str[0][c];
        in.s2nw = S.str[1][lnw];
        in.s3sse = S.str[2][lsse];
        in.s4sw = S.str[3][lsw];
        in.s5 = S.str[4][c];
        in.s6sse = S.str[5][lsse];
        in.s7nw = S.str[6][lnw];
        in.s8sw = S.str[7][lsw];
        const StepuOut o = stepu_point(in, p);
        a.u_out[off + c] = o.u;
        a.v_out[off + c] = o.v;
        if (kLast) {
          a.strintx[off + c] = o.strintx;
          a.strinty[off + c] = o.strinty;
          a.Cb[off + c] = o.Cb;
        }
      }
    }
    consumer_sync();  // stage s and the str table are free again
    if (c == 0) mbar_arrive(&S.empty[s]);
  }
}

size_t smem_bytes() { return sizeof(Smem) + 128; }

}  // namespace

int tma_prepare(int device) {
  const int bytes = (int)smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  (void)device;
  return e == cudaSuccess ? 0 : (int)e;
}

void launch_tma(const TmaArgs &a, const Params &p, bool last, int nctas, cudaStream_t st) {
  if (a.ntiles <= 0) return;
  const int grid = a.ntiles < nctas ? a.ntiles : nctas;
  if (last)
    k_tma<true><<<grid, kThreads, smem_bytes(), st>>>(a, p);
  else
    k_tma<false><<<grid, kThreads, smem_bytes(), st>>>(a, p);
}

}  // namespace evp
