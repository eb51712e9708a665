// evp_kernels_tma.cu -- the fused EVP subcycle as a persistent, TMA-fed
// producer/consumer kernel (sm_100a).
//
// CTA b works through the tiles of its run, t = run_off[b] .. run_off[b+1]-1,
// in order (one CTA per SM).  A tile's inputs are staged in shared memory in
// two parts with different lifetimes:
//   - the stress part (geometry, strength, packed index words, the 12
//     stresses, u and v of the owned points and of the stencil's extra
//     points, and the recomputed forward halo) is dead once stress is done;
//     it has a two-slot ring, so one later tile loads while one computes;
//   - the stepu part (the 13 stepu inputs) has one slot, loaded while the
//     consumers compute the tile's stress.
// The owned points of a tile are contiguous slots and its per-call constants
// one contiguous block, so the owned data arrive by cp.async.bulk (TMA)
// copies completing on the slot's mbarrier (complete_tx); the halo and the
// extra velocities are gathered with 4/8-byte cp.async, whose completion
// arrives on the same mbarrier (cp.async.mbarrier.arrive).
// Producer warps: the bulk warp (the bulk copies of both parts) and
// kGatherWarps gather warps issuing the cp.async gathers side by side with it.  The producers' own inputs -- the
// tile's slot range and gather lists -- are one 1.3 KB record per tile that a
// bulk copy brings kRecRing tiles ahead, so no producer waits on a global
// load.
// Eight consumer warps (one thread per compute-set point: the tile's owned
// points, then its forward halo, 256 at most) compute stress from shared
// memory into the tile's str table, then stepu for the owned points, writing
// the new stresses and velocities to the other ping-pong buffer.  Stepu reads
// str from the tile's own table and from the previous tile's, which stays
// alive: three str tables rotate, so that one tile's stress can start while
// stepu still reads the two before it.
//
// Every mbarrier wait is bounded by %globaltimer (kWaitNs): on expiry the
// kernel records an error code, every thread of the consumer group leaves the
// tile loop together, and each producer warp waits (bounded) for the copies it
// has issued before it exits, so nothing is left in flight.
#include <cstdint>

#include "evp_kernels.cuh"
#include "evp_tiles.h"

namespace evp {

namespace {

constexpr int kSSlots = 2;                          // stress-part ring
constexpr int kRecRing = 4;                         // producer records in flight
constexpr int kConsumers = kTileCompute;            // 256 = 8 warps, two per scheduler
constexpr int kGatherWarps = 2;                     // producer warps issuing cp.async gathers
constexpr int kStageWarps = 1 + kGatherWarps;       // bulk warp + gather warps
constexpr int kThreads = kConsumers + 32 * kStageWarps;
constexpr int kUV = kTileOwned + kTileUvx;
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s

// Stress part of a tile.
struct SSlot {
  double cs[kConstStressFields][kTileOwned];  // constant block fields 0..7 (one bulk copy)
  double s12[12][kTileOwned];                 // the 12 stresses
  double u[kUV];
  double v[kUV];
  double hf[kTmaStressFields][kTileHalo];  // halo: 6 geometry, strength, 12 stresses
  uint32_t hmeta[kTileHalo];
  uint32_t hlcc[kTileHalo];
  uint32_t hlcor[kTileHalo];
  int hdr[4];  // tile offset, owned count, halo count (written by the bulk warp)
};

// Stepu part of a tile: constant block fields 8..20 (one bulk copy).
struct USlot {
  double cu[kTmaStepuFields][kTileOwned];
};

static_assert(kConstTileSlots == kTileOwned, "constant blocks hold one tile");
static_assert(kConstFields == kConstStressFields + kTmaStepuFields, "constant block layout");

struct Smem {
  SSlot ss[kSSlots];
  USlot us;
  double str[3][8][kStrRow];  // rotating str tables; position kZeroSlot holds 0
  int32_t rec[kRecRing][kRecInts];
  unsigned long long sfull[kSSlots];
  unsigned long long sempty[kSSlots];
  unsigned long long ufull, uempty;
  unsigned long long rec_full[kRecRing];
  int abort_flag;
  int prod_ok;  // the bulk warp's waits succeeded for the current tile
};

static_assert(sizeof(SSlot) % 16 == 0 && sizeof(USlot) % 16 == 0,
              "slots must keep 16-byte alignment");
static_assert((kRecInts * 4) % 16 == 0, "records are bulk-copied");
static_assert(sizeof(Smem) <= 227 * 1024, "shared memory per block");

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

// Bounded wait for the phase of parity `parity` to complete; on expiry the
// wait's code goes into the error word.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity,
                                          int *err, int code,
                                          unsigned long long limit_ns = kWaitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) {
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

// Barrier of the consumer warps that also ORs a predicate over them.
__device__ __forceinline__ bool consumer_sync_or(bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(kConsumers)
      : "memory");
  return r != 0;
}

// The bulk warp and the gather warps.
__device__ __forceinline__ void stage_sync() {
  asm volatile("bar.sync 2, %0;" ::"r"(32 * kStageWarps) : "memory");
}

__device__ __forceinline__ void trace_stamp(const TmaArgs &a, int it, int slot) {
  if (a.trace && blockIdx.x == 0 && it < kTraceTiles) a.trace[it * 8 + slot] = (long long)global_ns();
}

// The stepu part of tile t (constant block fields 8..20) into the stepu slot.
__device__ __forceinline__ void issue_stepu(const TmaArgs &a, Smem &S, int t) {
  constexpr uint32_t kBytes = kTmaStepuFields * kTileOwned * 8u;
  mbar_arrive_expect_tx(&S.ufull, kBytes);
  bulk_g2s(S.us.cu, a.cblk + ((size_t)t * kConstFields + kConstStressFields) * kTileOwned, kBytes,
           &S.ufull);
}

// ---------------- the kernel ---------------------------------------------------
// kStd: parameters with std_params(p) (stress_update_std).
template <bool kLast, bool kStd>
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
    for (int s = 0; s < kSSlots; s++) {
      mbar_init(&S.sfull[s], 1 + 32 * kGatherWarps);  // expect_tx arrival + cp.async lanes
      mbar_init(&S.sempty[s], 1);                     // one consumer arrival per use
    }
    mbar_init(&S.ufull, 1);
    mbar_init(&S.uempty, kConsumers / 32);  // one arrival per consumer warp
    for (int r = 0; r < kRecRing; r++) mbar_init(&S.rec_full[r], 1);
    S.abort_flag = 0;
    mbar_fence_init();
  }
  if (tid < 24) S.str[tid >> 3][tid & 7][kZeroSlot] = 0.0;
  __syncthreads();

  const int T0 = a.run_off[blockIdx.x], T1 = a.run_off[blockIdx.x + 1];
  constexpr uint32_t kCsBytes = kConstStressFields * kTileOwned * 8u;
  constexpr size_t kBlk = (size_t)kConstFields * kTileOwned;  // doubles per constant block

  if (tid >= kConsumers) {
    // ======================= producers ===================================
    // The bulk warp (pw 0) waits for the tile record and the free slot,
    // writes the slot header, arms the slot's full barrier and issues the
    // bulk copies (TMA unit); the gather warps meanwhile issue the 8-byte
    // cp.async gathers of the forward halo and the extra velocities
    // (load/store path).  Two named-barrier handshakes per tile order the
    // warps: after the first the slot is armed and the record readable, after
    // the second every warp is done with the record, which the bulk warp then
    // refills.  The bulk warp's waits are bounded and it reaches the first
    // handshake on every path, so the handshakes cannot hang; a failed wait
    // is passed on through prod_ok.
    // The bulk warp also issues the stepu part: tile i's stress part goes
    // out two tiles ahead of its use, tile j's stepu part as soon as the
    // stepu slot is free (end of stepu(j-1)).  The TMA unit serves the
    // copies in issue order, so in round i the stepu part of tile i-2 is
    // issued before the stress part of tile i (whose slot was freed earlier,
    // at the end of stress(i-3)), which keeps the urgent copy at the front.
    const int pw = (tid - kConsumers) >> 5;
    const int lane = tid & 31;
    constexpr uint32_t kRecBytes = kRecInts * 4u;
    if (pw == 0 && lane == 0) {
      for (int r = 0; r < kRecRing; r++) {
        const int t = T0 + r;
        if (t >= T1) break;
        mbar_arrive_expect_tx(&S.rec_full[r], kRecBytes);
        bulk_g2s(S.rec[r], a.tile_rec + (size_t)t * kRecInts, kRecBytes, &S.rec_full[r]);
      }
    }
    int issued = 0;
    int nu = 0;  // stepu parts issued (counted by the bulk warp's lane 0)
    bool ok = true;
    for (int t = T0; t < T1; t++) {
      const int r = issued % kRecRing;
      const int s = issued % kSSlots;
      const uint32_t use = (uint32_t)(issued / kSSlots);
      SSlot &st = S.ss[s];
      const int32_t *rec = S.rec[r];
      if (pw == 0) {
        int w = 1;
        if (lane == 0) {
          w = mbar_wait(&S.rec_full[r], (uint32_t)(issued / kRecRing) & 1, a.err, 6) ? 1 : 0;
          trace_stamp(a, issued, 3);
          if (w && issued >= kSSlots) {
            // stepu part nu == issued - 2; its slot frees after stepu(nu - 1)
            w = mbar_wait(&S.uempty, (uint32_t)(nu - 1) & 1, a.err, 9) ? 1 : 0;
            if (w) issue_stepu(a, S, T0 + (nu++));
            if (w) w = mbar_wait(&S.sempty[s], (use - 1) & 1, a.err, 2) ? 1 : 0;
          }
          trace_stamp(a, issued, 4);
        }
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w) {
          const int nh = rec[3];
          for (int h = lane; h < nh; h += 32) {
            st.hlcor[h] = (uint32_t)rec[kRecHLcor + h];
            st.hlcc[h] = (uint32_t)rec[kRecHLcc + h];
          }
          if (lane == 0) {
            st.hdr[0] = rec[0];
            st.hdr[1] = rec[1];
            st.hdr[2] = nh;
          }
          __syncwarp();
          // release: the header and halo indices are visible to consumers
          // once the phase completes
          if (lane == 0) {
            const uint32_t b8 = (uint32_t)((rec[1] + 3) & ~3) * 8u;
            mbar_arrive_expect_tx(&S.sfull[s], kCsBytes + 14 * b8);
          }
        }
        if (lane == 0) S.prod_ok = w;
      }
      stage_sync();  // handshake 1
      if (!S.prod_ok) {
        ok = false;
        break;
      }
      const int off = rec[0], cnt = rec[1], nx = rec[2], nh = rec[3];
      if (pw == 0) {
        const uint32_t b8 = (uint32_t)((cnt + 3) & ~3) * 8u;
        if (lane == 0)
          bulk_g2s(st.cs, a.cblk + (size_t)t * kBlk, kCsBytes, &S.sfull[s]);
        else if (lane <= 12)
          bulk_g2s(st.s12[lane - 1], a.sf[6 + lane] + off, b8, &S.sfull[s]);
        else if (lane == 13)
          bulk_g2s(st.u, a.u_in + off, b8, &S.sfull[s]);
        else if (lane == 14)
          bulk_g2s(st.v, a.v_in + off, b8, &S.sfull[s]);
        if (lane == 0) {
          if (issued == 0) issue_stepu(a, S, T0 + (nu++));
          trace_stamp(a, issued, 6);
        }
      } else {
        // gather warp gw takes the velocity extras u (first) / v (last) and
        // every kGatherWarps-th halo field; the last one also the halo meta
        const int gw = pw - 1;
        if (gw == 0)
          for (int x = lane; x < nx; x += 32)
            cp_async8(&st.u[kTileOwned + x], a.u_in + rec[kRecUvx + x]);
        if (gw == kGatherWarps - 1)
          for (int x = lane; x < nx; x += 32)
            cp_async8(&st.v[kTileOwned + x], a.v_in + rec[kRecUvx + x]);
        for (int h = lane; h < nh; h += 32) {
          const int g = rec[kRecHalo + h];
          for (int f = gw; f < kTmaStressFields; f += kGatherWarps) cp_async8(&st.hf[f][h], a.sf[f] + g);
          if (gw == kGatherWarps - 1) cp_async4(&st.hmeta[h], a.meta + g);
        }
        cp_async_arrive(&S.sfull[s]);
        if (gw == 0 && lane == 0) trace_stamp(a, issued, 7);
      }
      // the record's generic reads come before its async-proxy refill
      fence_proxy_async();
      stage_sync();  // handshake 2
      if (pw == 0) {
        if (lane == 0) trace_stamp(a, issued, 0);
        const int tr = t + kRecRing;
        if (lane == 0 && tr < T1) {
          mbar_arrive_expect_tx(&S.rec_full[r], kRecBytes);
          bulk_g2s(S.rec[r], a.tile_rec + (size_t)tr * kRecInts, kRecBytes, &S.rec_full[r]);
        }
        if (a.prefetch > 0) {
          const int tp = t + a.prefetch;
          if (tp < T1 && lane < 15) {
            // what the stage load of a later tile copies: its constant block,
            // the owned ranges of the 12 stresses, u and v
            const int po = a.tile_meta[8 * tp], pc = a.tile_meta[8 * tp + 1];
            const uint32_t pb = (uint32_t)((pc + 3) & ~3) * 8u;
            if (lane == 0)
              bulk_prefetch_l2(a.cblk + (size_t)tp * kBlk, (uint32_t)(kBlk * 8u));
            else if (lane <= 12)
              bulk_prefetch_l2(a.sf[6 + lane] + po, pb);
            else
              bulk_prefetch_l2((lane == 13 ? a.u_in : a.v_in) + po, pb);
          }
        }
      }
      issued++;
    }
    if (pw == 0) {
      if (ok && lane == 0) {
        // the stepu parts of the last tiles
        for (; nu < issued; nu++) {
          if (!mbar_wait(&S.uempty, (uint32_t)(nu - 1) & 1, a.err, 9)) break;
          issue_stepu(a, S, T0 + nu);
        }
      }
      if (lane == 0 && nu > 0) mbar_wait(&S.ufull, (uint32_t)(nu - 1) & 1, a.err, 10);
      if (!ok) {
        // Consumers stopped early: wait (bounded) until every issued slot has
        // landed so that no copy targets shared memory after the CTA exits.
        for (int k = issued - kSSlots; k < issued; k++) {
          if (k < 0) continue;
          if (lane == 0) mbar_wait(&S.sfull[k % kSSlots], (uint32_t)(k / kSSlots) & 1, a.err, 3);
        }
      }
      // records issued ahead and never consumed must land before exit too
      if (lane == 0) {
        for (int k = issued; k < issued + kRecRing; k++) {
          const int t = T0 + k;
          if (t >= T1) break;
          mbar_wait(&S.rec_full[k % kRecRing], (uint32_t)(k / kRecRing) & 1, a.err, 7);
        }
      }
    }
    __syncwarp();
    return;
  }

  // ========================= consumers ===================================
  // Per tile one block barrier: after stress, when the tile's str table is
  // complete.  Stepu then runs warp by warp and each warp goes straight on to
  // the next tile's stress, so one warp's stepu overlaps the others' stress.
  // Stepu of tile k reads the tables of tiles k and k-1 while stress of tile
  // k+1 writes the third; the table it writes last held tile k-2, whose
  // readers (stepu of k-2 and k-1) every warp has finished before any passes
  // the barrier of tile k.  The stepu slot is released by one arrival per
  // warp.  A wait that ran out anywhere is OR-reduced at the barrier, so all
  // consumers leave the loop together.
  const int c = tid;  // compute-set index: owned c < cnt, halo cnt + h
  const int lane = tid & 31;
  bool fail = false;
  int it = 0;
  for (int t = T0; t < T1; t++, it++) {
    const int s = it % kSSlots;
    const int b = it % 3;
    const int bp = (it + 2) % 3;  // the previous tile's table
    const bool have = mbar_wait(&S.sfull[s], (uint32_t)(it / kSSlots) & 1, a.err, 1);
    fail |= !have;
    if (tid == 0) trace_stamp(a, it, 1);
    const SSlot &st = S.ss[s];

    // ---------------- phase 1: stress ------------------------------------
    // The owned thread keeps what stepu needs from the stress part (its
    // index word and velocity) so that the slot can be released after stress.
    uint32_t m = 0;
    double uold = 0.0, vold = 0.0;
    int off = 0, cnt = 0;
    if (have) {
      off = st.hdr[0];
      cnt = st.hdr[1];
      const int nh = st.hdr[2];
      const bool own = c < cnt;
      const int h = c - cnt;
      if (own || h < nh) {
        uint32_t lc;
        if (own) {
          const unsigned long long ml = (unsigned long long)__double_as_longlong(st.cs[7][c]);
          m = (uint32_t)ml;
          lc = (uint32_t)(ml >> 32);
          uold = st.u[c];
          vold = st.v[c];
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
          const double *F = own ? &st.cs[0][c] : &st.hf[0][h];
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
          if (kStd)
            stress_update_std(s12, out, sr, F[6 * fs], gm, p);
          else
            stress_update(s12, out, sr, F[6 * fs], gm, p);
          if (own) {
#pragma unroll
            for (int k = 0; k < 12; k++) a.s_out[k][off + c] = s12[k];
          }
        }
#pragma unroll
        for (int k = 0; k < 8; k++) S.str[b][k][c] = out[k];
        if (kLast && own) {
#pragma unroll
          for (int k = 0; k < 8; k++) a.str_out[k][off + c] = out[k];
        }
      }
    }
    // str of this tile complete; the stress part of slot s is free again
    const bool stop = consumer_sync_or(fail);
    if (tid == 0) {
      trace_stamp(a, it, 2);
      mbar_arrive(&S.sempty[s]);
    }
    if (stop) break;

    // ---------------- phase 2: stepu on owned points, warp by warp ----------
    const bool hu = mbar_wait(&S.ufull, (uint32_t)it & 1, a.err, 11);
    fail |= !hu;
    if (hu && c < cnt && !((m >> 30) & kSkipU)) {
      const USlot &us = S.us;
      const double(&str)[8][kStrRow] = S.str[b];
      // a neighbour's str: own table, or the previous tile's (kStrPrev)
      const uint32_t vnw = m & kLnbMask, vsw = (m >> kLnbBits) & kLnbMask;
      const uint32_t vsse = (m >> (2 * kLnbBits)) & kLnbMask;
      const double(&tnw)[8][kStrRow] = (vnw & kStrPrev) ? S.str[bp] : S.str[b];
      const double(&tsw)[8][kStrRow] = (vsw & kStrPrev) ? S.str[bp] : S.str[b];
      const double(&tsse)[8][kStrRow] = (vsse & kStrPrev) ? S.str[bp] : S.str[b];
      const int lnw = vnw & (kStrPrev - 1), lsw = vsw & (kStrPrev - 1);
      const int lsse = vsse & (kStrPrev - 1);
      StepuIn in;
      in.uold = uold;
      in.vold = vold;
      in.kvrel = us.cu[0][c];
      in.uocn = us.cu[1][c];
      in.vocn = us.cu[2][c];
      in.waterx = us.cu[3][c];
      in.watery = us.cu[4][c];
      in.forcex = us.cu[5][c];
      in.forcey = us.cu[6][c];
      in.umassdti = us.cu[7][c];
      in.fm = us.cu[8][c];
      in.uarear = us.cu[9][c];
      in.Tbu = us.cu[10][c];
      in.uinit = us.cu[11][c];
      in.vinit = us.cu[12][c];
      in.s1 = str[0][c];
      in.s2nw = tnw[1][lnw];
      in.s3sse = tsse[2][lsse];
      in.s4sw = tsw[3][lsw];
      in.s5 = str[4][c];
      in.s6sse = tsse[5][lsse];
      in.s7nw = tnw[6][lnw];
      in.s8sw = tsw[7][lsw];
      const StepuOut o = stepu_point(in, p);
      a.u_out[off + c] = o.u;
      a.v_out[off + c] = o.v;
      if (kLast) {
        a.strintx[off + c] = o.strintx;
        a.strinty[off + c] = o.strinty;
        a.Cb[off + c] = o.Cb;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&S.uempty);  // this warp is done with the stepu slot
    if (tid == 0) trace_stamp(a, it, 5);
  }
}

size_t smem_bytes() { return sizeof(Smem); }

// One thread waits, through the kernel's own bounded wait, on an mbarrier at
// which nothing ever arrives: the wait runs out after limit_ns and records
// kProbeCode, as a timed-out wait of the subcycle kernel would.
constexpr int kProbeCode = 12;

__global__ void k_wait_probe(int *err, unsigned long long limit_ns) {
  __shared__ unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
    mbar_wait(&bar, 0, err, kProbeCode, limit_ns);
  }
}

}  // namespace

const char *tma_wait_name(int code) {
  switch (code) {
    case 1: return "a consumer waited for a tile's stress inputs";
    case 2: return "the producer waited for a free stress slot";
    case 3: return "the producer waited for its copies to land after an early stop";
    case 6: return "the producer waited for a tile record";
    case 7: return "the producer waited for records issued ahead";
    case 8: return "the dynamic shared memory was not 16-byte aligned";
    case 9: return "the producer waited for the stepu slot";
    case 10: return "the producer waited for its last stepu copy";
    case 11: return "a consumer waited for a tile's stepu inputs";
    case kProbeCode: return "the wait probe (evp1d_debug_wait_timeout)";
    default: return "unknown";
  }
}

cudaError_t tma_binary_version(int *version) {
  cudaFuncAttributes at;
  const cudaError_t e = cudaFuncGetAttributes(&at, k_tma<false, true>);
  if (e == cudaSuccess) *version = at.binaryVersion;
  return e;
}

void launch_wait_probe(int *err, unsigned long long limit_ns, cudaStream_t st) {
  k_wait_probe<<<1, 32, 0, st>>>(err, limit_ns);
}

int tma_prepare(int device) {
  const int bytes = (int)smem_bytes();
  void (*const ks[4])(TmaArgs, Params) = {k_tma<false, false>, k_tma<true, false>,
                                          k_tma<false, true>, k_tma<true, true>};
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 4 && e == cudaSuccess; i++)
    e = cudaFuncSetAttribute(ks[i], cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  (void)device;
  return e == cudaSuccess ? 0 : (int)e;
}

void launch_tma(const TmaArgs &a, const Params &p, bool last, cudaStream_t st) {
  if (a.ntiles <= 0 || a.nruns <= 0) return;
  const int grid = a.nruns;
  const bool std = std_params(p);
  if (last && std)
    k_tma<true, true><<<grid, kThreads, smem_bytes(), st>>>(a, p);
  else if (last)
    k_tma<true, false><<<grid, kThreads, smem_bytes(), st>>>(a, p);
  else if (std)
    k_tma<false, true><<<grid, kThreads, smem_bytes(), st>>>(a, p);
  else
    k_tma<false, false><<<grid, kThreads, smem_bytes(), st>>>(a, p);
}

}  // namespace evp
