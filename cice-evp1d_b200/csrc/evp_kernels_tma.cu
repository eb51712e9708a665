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
// The producer's own inputs -- the tile's slot range and gather lists -- are
// one 1.3 KB record per tile that a bulk copy brings kRecRing tiles ahead,
// so the producer never waits on a global load.
// Ten consumer warps (one thread per compute-set point: 256 owned + 64 halo)
// compute stress from shared memory into the shared str table, then stepu for
// the owned points, writing the new stresses and velocities to the other
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
constexpr int kRecRing = 4;                         // producer records in flight
constexpr int kConsumers = kTileOwned + kTileHalo;  // 320 = 10 warps
constexpr int kThreads = kConsumers + 32;           // + 1 producer warp
constexpr int kUV = kTileOwned + kTileUvx;
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s

struct Stage {
  double cf[kConstFields][kTileOwned];  // the tile's constant block (one bulk copy)
  double s12[12][kTileOwned];           // the 12 stresses
  double u[kUV];
  double v[kUV];
  double hf[kTmaStressFields][kTileHalo];  // halo: 6 geometry, strength, 12 stresses
  uint32_t hmeta[kTileHalo];
  uint32_t hlcc[kTileHalo];
  uint32_t hlcor[kTileHalo];
  int hdr[4];  // tile offset, owned count, halo count (written by the producer)
};

static_assert(kConstTileSlots == kTileOwned, "constant blocks hold one tile");
static_assert(kConstFields == 7 + kTmaStepuFields + 1, "constant block layout");

struct Smem {
  Stage st[kStages];
  double str[8][kZeroSlot + 2];
  int32_t rec[kRecRing][kRecInts];
  unsigned long long full[kStages];
  unsigned long long empty[kStages];
  unsigned long long rec_full[kRecRing];
  int abort_flag;
};

static_assert(sizeof(Stage) % 16 == 0, "stage must keep 16-byte alignment");
static_assert((kRecInts * 4) % 16 == 0, "records are bulk-copied");

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

// Bulk prefetch of global memory into L2 (no shared memory, no completion).
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
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

// Order this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) accesses to the same memory.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void consumer_sync() {
  asm volatile("bar.sync 1, %0;" ::"r"(kConsumers) : "memory");
}

__device__ __forceinline__ void trace_stamp(const TmaArgs &a, int it, int slot) {
  if (a.trace && blockIdx.x == 0 && it < kTraceTiles) a.trace[it * 8 + slot] = (long long)global_ns();
}

// ---------------- the kernel ---------------------------------------------------
template <bool kLast>
__global__ void __launch_bounds__(kThreads, 1) k_tma(TmaArgs a, Params p) {
  // Indexed straight off the __shared__ symbol (no integer round trip), so
  // every access compiles to a shared-memory load or store, not a generic one.
  // The bulk copies need 16-byte alignment, which the dynamic shared memory
  // base has (checked: a misaligned base is refused, not faulted on).
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &S = *reinterpret_cast<Smem *>(smem_raw);
  const int tid = threadIdx.x;
  if (smem_addr(smem_raw) & 15u) {
    if (tid == 0) atomicMax(a.err, 8);
    return;
  }
  if (tid == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&S.full[s], 1 + 32);  // expect_tx arrival + 32 cp.async lanes
      mbar_init(&S.empty[s], 1);      // one consumer arrival per use
    }
    for (int r = 0; r < kRecRing; r++) mbar_init(&S.rec_full[r], 1);
    S.abort_flag = 0;
    mbar_fence_init();
  }
  if (tid < 8) S.str[tid][kZeroSlot] = 0.0;
  __syncthreads();

  if (tid >= kConsumers) {
    // ======================= producer warp ==============================
    const int lane = tid - kConsumers;
    const int T0 = blockIdx.x, dT = gridDim.x;
    constexpr uint32_t kRecBytes = kRecInts * 4u;
    if (lane == 0) {
      for (int r = 0; r < kRecRing; r++) {
        const int t = T0 + r * dT;
        if (t >= a.ntiles) break;
        mbar_arrive_expect_tx(&S.rec_full[r], kRecBytes);
        bulk_g2s(S.rec[r], a.tile_rec + (size_t)t * kRecInts, kRecBytes, &S.rec_full[r]);
      }
    }
    int issued = 0;
    bool ok = true;
    for (int t = T0; t < a.ntiles; t += dT) {
      const int r = issued % kRecRing;
      int w = 1;
      if (lane == 0) w = mbar_wait(&S.rec_full[r], (uint32_t)(issued / kRecRing) & 1, a.err, 6);
      const int s = issued % kStages;
      const uint32_t use = (uint32_t)(issued / kStages);
      if (w && issued >= kStages && lane == 0)
        w = mbar_wait(&S.empty[s], (use - 1) & 1, a.err, 2) ? 1 : 0;
      w = __shfl_sync(0xffffffffu, w, 0);
      if (!w) {
        ok = false;
        break;
      }
      const int32_t *rec = S.rec[r];
      const int off = rec[0], cnt = rec[1], nx = rec[2], nh = rec[3];
      Stage &st = S.st[s];
      for (int h = lane; h < nh; h += 32) {
        st.hlcor[h] = (uint32_t)rec[kRecHLcor + h];
        st.hlcc[h] = (uint32_t)rec[kRecHLcc + h];
      }
      if (lane == 0) {
        st.hdr[0] = off;
        st.hdr[1] = cnt;
        st.hdr[2] = nh;
      }
      __syncwarp();
      const uint32_t n4 = (uint32_t)((cnt + 3) & ~3);
      const uint32_t b8 = n4 * 8u;
      constexpr uint32_t kConstBytes = kConstFields * kTileOwned * 8u;
      // release: the header and halo indices are visible to consumers once
      // the phase completes
      if (lane == 0) mbar_arrive_expect_tx(&S.full[s], kConstBytes + 14 * b8);
      __syncwarp();
      if (lane == 0)
        bulk_g2s(st.cf, a.cblk + (size_t)t * kConstFields * kTileOwned, kConstBytes, &S.full[s]);
      else if (lane <= 12)
        bulk_g2s(st.s12[lane - 1], a.sf[6 + lane] + off, b8, &S.full[s]);
      else if (lane == 13)
        bulk_g2s(st.u, a.u_in + off, b8, &S.full[s]);
      else if (lane == 14)
        bulk_g2s(st.v, a.v_in + off, b8, &S.full[s]);
      for (int x = lane; x < nx; x += 32) {
        const int g = rec[kRecUvx + x];
        cp_async8(&st.u[kTileOwned + x], a.u_in + g);
        cp_async8(&st.v[kTileOwned + x], a.v_in + g);
      }
      for (int h = lane; h < nh; h += 32) {
        const int g = rec[kRecHalo + h];
        for (int f = 0; f < kTmaStressFields; f++) cp_async8(&st.hf[f][h], a.sf[f] + g);
        cp_async4(&st.hmeta[h], a.meta + g);
      }
      cp_async_arrive(&S.full[s]);
      if (lane == 0) trace_stamp(a, issued, 0);
      // record slot r has been read: refill it kRecRing tiles ahead
      fence_proxy_async();
      __syncwarp();
      const int tr = t + kRecRing * dT;
      if (lane == 0 && tr < a.ntiles) {
        mbar_arrive_expect_tx(&S.rec_full[r], kRecBytes);
        bulk_g2s(S.rec[r], a.tile_rec + (size_t)tr * kRecInts, kRecBytes, &S.rec_full[r]);
      }
      if (a.prefetch > 0) {
        const int tp = t + a.prefetch * dT;
        if (tp < a.ntiles && lane < 2) {
          // the owned slot range of every staged field of a later tile
          const int po = a.tile_meta[8 * tp], pc = a.tile_meta[8 * tp + 1];
          const uint32_t pn = (uint32_t)((pc + 3) & ~3);
          for (int f = lane; f < kTmaStressFields; f += 2) bulk_prefetch_l2(a.sf[f] + po, pn * 8u);
          for (int f = lane; f < kTmaStepuFields; f += 2) bulk_prefetch_l2(a.uf[f] + po, pn * 8u);
        }
      }
      issued++;
    }
    if (!ok) {
      // Consumers stopped early: wait (bounded) until every issued stage has
      // landed so that no copy targets shared memory after the CTA exits.
      for (int k = issued - kStages; k < issued; k++) {
        if (k < 0) continue;
        if (lane == 0) mbar_wait(&S.full[k % kStages], (uint32_t)(k / kStages) & 1, a.err, 3);
      }
    }
    // records issued ahead and never consumed must land before exit too
    if (lane == 0) {
      for (int k = issued; k < issued + kRecRing; k++) {
        const int t = T0 + k * dT;
        if (t >= a.ntiles) break;
        mbar_wait(&S.rec_full[k % kRecRing], (uint32_t)(k / kRecRing) & 1, a.err, 7);
      }
    }
    __syncwarp();
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
    if (tid == 0) trace_stamp(a, it, 1);
    const Stage &st = S.st[s];
    const int off = st.hdr[0], cnt = st.hdr[1], nh = st.hdr[2];

    // ---------------- phase 1: stress ------------------------------------
    const bool own = c < kTileOwned;
    const int h = c - kTileOwned;
    if (own ? c < cnt : h < nh) {
      uint32_t m, lc;
      if (own) {
        const unsigned long long ml = (unsigned long long)__double_as_longlong(st.cf[20][c]);
        m = (uint32_t)ml;
        lc = (uint32_t)(ml >> 32);
      } else {
        m = st.hmeta[h];
        lc = st.hlcor[h];
      }
      double out[8];
      if ((m >> 30) & kSkipT) {
#pragma unroll
        for (int k = 0; k < 8; k++) out[k] = 0.0;
      } else {
        // geometry and strength (fields 0..6), then the 12 stresses
        const double *F = own ? &st.cf[0][c] : &st.hf[0][h];
        const double *F12 = own ? &st.s12[0][c] : &st.hf[7][h];
        const int fs = own ? kTileOwned : kTileHalo;
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
        for (int k = 0; k < 12; k++) s12[k] = F12[k * fs];
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
    if (tid == 0) trace_stamp(a, it, 2);

    // ---------------- phase 2: stepu on owned points ------------------------
    if (c < cnt) {
      const uint32_t m = (uint32_t)__double_as_longlong(st.cf[20][c]);
      if (!((m >> 30) & kSkipU)) {
        const int lnw = m & kLnbMask, lsw = (m >> kLnbBits) & kLnbMask;
        const int lsse = (m >> (2 * kLnbBits)) & kLnbMask;
        StepuIn in;
        in.uold = st.u[c];
        in.vold = st.v[c];
        in.kvrel = st.cf[7][c];
        in.uocn = st.cf[8][c];
        in.vocn = st.cf[9][c];
        in.waterx = st.cf[10][c];
        in.watery = st.cf[11][c];
        in.forcex = st.cf[12][c];
        in.forcey = st.cf[13][c];
        in.umassdti = st.cf[14][c];
        in.fm = st.cf[15][c];
        in.uarear = st.cf[16][c];
        in.Tbu = st.cf[17][c];
        in.uinit = st.cf[18][c];
        in.vinit = st.cf[19][c];
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
    if (tid == 0) {
      trace_stamp(a, it, 5);
      mbar_arrive(&S.empty[s]);
    }
  }
}

size_t smem_bytes() { return sizeof(Smem); }

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
