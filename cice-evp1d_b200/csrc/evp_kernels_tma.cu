// evp_kernels_tma.cu -- the fused EVP subcycle as a TMA-fed producer/consumer
// kernel (sm_100a), one CTA per SM.
//
// CTA b works through the tiles of its run, t = run_off[b] .. run_off[b+1]-1,
// in order.  A tile's stress inputs (geometry, strength, packed index words,
// the 12 stresses, u and v of the owned points and of the stencil's extra
// points, and the recomputed forward halo) are staged in shared memory in a
// two-slot ring, so one later tile loads while one computes.  The owned
// points of a tile are contiguous slots and its per-call constants one
// contiguous block, so the owned data arrive by cp.async.bulk (TMA) copies
// completing on the slot's mbarrier (complete_tx); the halo and the extra
// velocities are gathered with 4/8-byte cp.async, whose completion arrives on
// the same mbarrier (cp.async.mbarrier.arrive).
// Producer warps: the bulk warp (the bulk copies) and kGatherWarps gather
// warps issuing the cp.async gathers side by side with it.  The producers'
// own inputs -- the tile's slot range and gather lists -- are one 1.3 KB
// record per tile that a bulk copy brings kRecRing tiles ahead, so no
// producer waits on a global load.
// Eight consumer warps (one thread per compute-set point: the tile's owned
// points, then its forward halo, 256 at most) compute stress from shared
// memory into the tile's str table, then stepu for the owned points, writing
// the new stresses and velocities to the other ping-pong buffer.  Stepu reads
// str from the tile's own table and from the previous tile's, which stays
// alive: three str tables rotate, so that one tile's stress can start while
// stepu still reads the two before it.  The 13 stepu inputs of a tile (the
// second part of its constant block) arrive by one more bulk copy into a
// stepu slot, which the consumers release as soon as each has its point's
// inputs in registers.  Where every Tbu of the call is +0, every uinit and
// vinit finite and revp == 0, the part stops after its tenth field: Tbu is
// +0, and revp*uinit a signed zero whose sign comes from the packed word.
// Consecutive one-subcycle launches overlap: each CTA lets the next launch
// start at once (griddepcontrol.launch_dependents), and a launch started that
// way loads its first tile's records, constants and stepu part while the
// previous one finishes, reading the state only after griddepcontrol.wait.
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

static_assert(kConstTileSlots == kTileOwned, "constant blocks hold one tile");
static_assert(kConstFields == kConstStressFields + kTmaStepuFields, "constant block layout");

// Stepu part of a tile: constant block fields 8..20 (one bulk copy).
struct USlot {
  double cu[kTmaStepuFields][kTileOwned];
};

struct Smem {
  SSlot ss[kSSlots];
  USlot us;
  double str[3][8][kStrRow];  // rotating str tables; position kZeroSlot holds 0
  int32_t rec[kRecRing][kRecInts];
  unsigned long long sfull[kSSlots];
  unsigned long long sempty[kSSlots];
  unsigned long long rec_full[kRecRing];
  unsigned long long ufull, uempty;
  int abort_flag;
  int prod_ok;  // the bulk warp's waits succeeded for the current tile
};

static_assert(sizeof(SSlot) % 16 == 0, "slots must keep 16-byte alignment");
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

// Non-blocking test whether the phase of parity `parity` has completed.
__device__ __forceinline__ bool mbar_test_wait(unsigned long long *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
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

// Acquire load of a counter another CTA raises (gpu scope).
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Order this thread's generic-proxy global accesses with its async-proxy
// (bulk copy) accesses of global memory.
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void fence_acq_rel_gpu() {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}

// Bounded wait until the counter *e, which other CTAs raise, reaches `need`
// (acquire); on expiry the wait's code goes into the error word.
__device__ __forceinline__ bool wait_counter(const unsigned *e, unsigned need, int *err,
                                             int code, unsigned long long limit_ns) {
  if (ld_acquire(e) >= need) return true;
  const unsigned long long t0 = global_ns();
  while (ld_acquire(e) < need) {
    if (global_ns() - t0 > limit_ns) {
      atomicMax(err, code);
      return false;
    }
  }
  return true;
}

// Relaxed load of a counter another CTA raises (gpu scope, past L1).
__device__ __forceinline__ unsigned ld_relaxed(const unsigned *p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Coherent 8-byte load (at L2) of state other CTAs may have written.
__device__ __forceinline__ double ld_cg(const double *p) { return __ldcg(p); }

// ---------------- the kernel ---------------------------------------------------
// kStd: parameters with std_params(p) (stress_update_std).  The launch runs
// a.nsub subcycles; CTA b works through its run's tiles once per subcycle.
// kMulti: a launch of several subcycles (a.nsub > 1 with per-tile counters);
// otherwise one subcycle, whose last-subcycle outputs kLast selects.
template <bool kLast, bool kStd, bool kMulti>
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
    for (int r = 0; r < kRecRing; r++) mbar_init(&S.rec_full[r], 1);
    mbar_init(&S.ufull, 1);
    mbar_init(&S.uempty, kConsumers / 32);  // one arrival per consumer warp
    S.abort_flag = 0;
    mbar_fence_init();
  }
  if (tid < 24) S.str[tid >> 3][tid & 7][kZeroSlot] = 0.0;
  __syncthreads();
  // A launch of one subcycle may be followed by the next subcycle's, launched
  // as a programmatic dependent (a.pdl there): it can start as soon as every
  // CTA here has started.  Its CTAs cannot share an SM with these (shared
  // memory), so they take the SMs these CTAs leave, and before their
  // griddep_wait they read only what no subcycle writes (tile records,
  // constant blocks).
  if (!kMulti) griddep_launch_dependents();
  // the short stepu part (kTmaStepuCompact fields) where the call allows it
  const bool cpt = a.compact && __ldg(a.cflags) == 0;

  const int T0 = a.run_off[blockIdx.x], T1 = a.run_off[blockIdx.x + 1];
  const int n = T1 - T0;             // tiles of the run
  const int nq = kMulti ? n * a.nsub : n;  // (subcycle, tile) steps of the launch
  constexpr bool multi = kMulti;
  constexpr uint32_t kCsBytes = kConstStressFields * kTileOwned * 8u;
  constexpr size_t kBlk = (size_t)kConstFields * kTileOwned;  // doubles per constant block
  if (n <= 0) return;

  if (tid >= kConsumers) {
    // ======================= producers ===================================
    // The bulk warp (pw 0) waits for the tile record and the free slot,
    // writes the slot header, arms the slot's full barrier and issues the
    // bulk copies (TMA unit); the gather warps meanwhile gather the forward
    // halo and the extra velocities (8-byte cp.async, or, in a launch of
    // several subcycles, coherent loads).  Two named-barrier handshakes per
    // step order the warps: after the first the slot is armed and the record
    // readable, after the second every warp is done with the record, which
    // the bulk warp then refills.  The bulk warp's waits are bounded and it
    // reaches the first handshake on every path, so the handshakes cannot
    // hang; a failed wait is passed on through prod_ok.
    // Step q = (subcycle q / n, tile q % n).  In round q the bulk warp first
    // issues step q-1's stepu part (once stepu of step q-2 has freed the
    // stepu slot), then step q's stress part (once stress of step q-2 has
    // freed its slot).  The TMA unit serves copies in issue order, which keeps
    // the part needed first at the front.
    // A launch of several subcycles: step q's stress part goes out only when
    // every tile its tile depends on has finished the previous subcycle.  Its
    // lanes read those tiles' counters (relaxed) at the end of round q-1 and
    // check them here, so the check usually costs no wait; the acquire fence
    // then orders the state reads after the counters.  The bulk warp also
    // publishes this CTA's steps: once stepu of a step is done (all consumer
    // warps arrived on the stepu slot's barrier), it raises the tile's
    // counter after a gpu-scope fence, at the end of a round, where the wait
    // for the next slot absorbs the fence.  Every step's stepu part is out
    // before a round can wait on counters, so consumers finish every earlier
    // step without this round: no wait can depend on itself.
    const int pw = (tid - kConsumers) >> 5;
    const int lane = tid & 31;
    constexpr uint32_t kRecBytes = kRecInts * 4u;
    const uint32_t ubytes = (cpt ? kTmaStepuCompact : kTmaStepuFields) * kTileOwned * 8u;
    auto issue_stepu = [&](int q) {  // lane 0 of the bulk warp
      mbar_arrive_expect_tx(&S.ufull, ubytes);
      bulk_g2s(S.us.cu,
               a.cblk + ((size_t)(T0 + (kMulti ? q % n : q)) * kConstFields + kConstStressFields) *
                            kTileOwned,
               ubytes, &S.ufull);
    };
    int pub = 0;  // steps whose counters are raised (multi-subcycle launches)
    int nu = 0;   // stepu parts issued (the bulk warp's lane 0 counts)
    // Lane 0: raise the counters of every step whose stepu has completed.
    // Stepu phases below nu - 1 are known complete (the bulk warp waited for
    // each before issuing a later stepu part); phase nu - 1, the last one
    // issued, is tested: its parity is unambiguous because the phase after it
    // cannot complete before the next part goes out.
    auto publish = [&](int limit) {
      bool any = false;
      while (pub < limit) {
        const bool done = pub < nu - 1 || (pub == nu - 1 && mbar_test_wait(&S.uempty, (uint32_t)pub & 1));
        if (!done) break;
        if (!any) __threadfence();
        any = true;
        atomicAdd(a.epoch + T0 + (kMulti ? pub % n : pub), 1u);
        pub++;
      }
    };
    if (pw == 0 && lane == 0) {
      for (int r = 0; r < kRecRing && r < nq; r++) {
        const int t = T0 + (kMulti ? r % n : r);
        mbar_arrive_expect_tx(&S.rec_full[r], kRecBytes);
        bulk_g2s(S.rec[r], a.tile_rec + (size_t)t * kRecInts, kRecBytes, &S.rec_full[r]);
      }
    }
    int issued = 0;
    bool ok = true;
    unsigned seen = 0u;  // per lane: the smallest counter polled for the next step
    for (int q = 0; q < nq; q++) {
      const int sub = kMulti ? q / n : 0, t = T0 + (kMulti ? q % n : q);
      const int from = sub & 1;
      const double *u_in = kMulti && a.uv_step ? a.u[0] + (size_t)sub * a.uv_step : a.u[from];
      const double *v_in = kMulti && a.uv_step ? a.v[0] + (size_t)sub * a.uv_step : a.v[from];
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
            // step q-1's stepu part; the slot frees after stepu of step q-2
            w = mbar_wait(&S.uempty, (uint32_t)(nu - 1) & 1, a.err, 9) ? 1 : 0;
            if (w) issue_stepu(nu++);
            if (w) w = mbar_wait(&S.sempty[s], (use - 1) & 1, a.err, 2) ? 1 : 0;
          }
        }
        w = __shfl_sync(0xffffffffu, w, 0);
        if constexpr (kMulti) {
          if (w && sub > 0) {
            // the tiles step q depends on have finished subcycle sub - 1; the
            // warp waits together, lane 0 publishing this CTA's finished steps
            // meanwhile (a tile may wait on its own run's steps)
            const unsigned need = (unsigned)sub;
            const int d0 = a.dep_off[t], d1 = a.dep_off[t + 1];
            const unsigned long long t0 = global_ns();
            for (bool first = true;; first = false) {
              bool mine = true;
              for (int d = d0 + lane; d < d1 && mine; d += 32) {
                if (first && d < d0 + 32 && seen >= need) continue;
                mine = ld_relaxed(a.epoch + a.dep_idx[d]) >= need;
              }
              if (__all_sync(0xffffffffu, mine)) break;
              if (lane == 0) publish(q);
              // one decision for the whole warp (lane 0's clock)
              if (__shfl_sync(0xffffffffu, global_ns() - t0 > kWaitNs ? 1 : 0, 0)) {
                if (lane == 0) atomicMax(a.err, 13);
                w = 0;
                break;
              }
            }
            // acquire: the neighbours' state is read after their counters, by
            // these bulk copies (async proxy) and by the gather warps
            fence_acq_rel_gpu();
            fence_proxy_async_global();
          }
        }
        if (lane == 0) trace_stamp(a, issued, 4);
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
        if (lane == 0) {
          bulk_g2s(st.cs, a.cblk + (size_t)t * kBlk, kCsBytes, &S.sfull[s]);
          // a programmatic dependent has the time: the first stepu part
          // goes out before the state, while the previous launch drains
          if (issued == 0 && a.pdl) issue_stepu(nu++);
        }
        // the state the previous subcycle wrote
        if (issued == 0) griddep_wait();
        if (lane >= 1 && lane <= 12)
          bulk_g2s(st.s12[lane - 1], a.s[from][lane - 1] + off, b8, &S.sfull[s]);
        else if (lane == 13)
          bulk_g2s(st.u, u_in + off, b8, &S.sfull[s]);
        else if (lane == 14)
          bulk_g2s(st.v, v_in + off, b8, &S.sfull[s]);
        if (lane == 0) {
          if (issued == 0 && nu == 0) issue_stepu(nu++);
          trace_stamp(a, issued, 6);
        }
      } else {
        // gather warp gw takes the velocity extras u (first) / v (last) and
        // every kGatherWarps-th halo field; the last one also the halo meta
        const int gw = pw - 1;
        if (issued == 0) griddep_wait();
        if (!multi) {
          if (gw == 0)
            for (int x = lane; x < nx; x += 32)
              cp_async8(&st.u[kTileOwned + x], u_in + rec[kRecUvx + x]);
          if (gw == kGatherWarps - 1)
            for (int x = lane; x < nx; x += 32)
              cp_async8(&st.v[kTileOwned + x], v_in + rec[kRecUvx + x]);
          for (int h = lane; h < nh; h += 32) {
            const int g = rec[kRecHalo + h];
            for (int f = gw; f < kTmaStressFields; f += kGatherWarps)
              cp_async8(&st.hf[f][h], (f < 7 ? a.sg[f] : a.s[from][f - 7]) + g);
            if (gw == kGatherWarps - 1) cp_async4(&st.hmeta[h], a.meta + g);
          }
          cp_async_arrive(&S.sfull[s]);
        } else {
          // state written by other CTAs in this launch: loads at L2 (not a
          // copy that an earlier read may have left in this SM's L1)
          // Each lane issues a batch of loads before it stores any of them,
          // so that they overlap instead of taking one L2 round trip each.
          constexpr int kXPer = kTileUvx / 32;  // extras per lane at most
          for (int c = 0; c < 2; c++) {
            if (c == 0 ? gw != 0 : gw != kGatherWarps - 1) continue;
            const double *src = c == 0 ? u_in : v_in;
            double *dst = (c == 0 ? st.u : st.v) + kTileOwned;
            double xv[kXPer];
#pragma unroll
            for (int i = 0; i < kXPer; i++) {
              const int x = lane + 32 * i;
              xv[i] = x < nx ? ld_cg(src + rec[kRecUvx + x]) : 0.0;
            }
#pragma unroll
            for (int i = 0; i < kXPer; i++)
              if (lane + 32 * i < nx) dst[lane + 32 * i] = xv[i];
          }
          // halo: this warp's fields f = gw (mod kGatherWarps) of every halo
          // point, spread over the lanes by (point, field)
          const int nf = (kTmaStressFields - gw + kGatherWarps - 1) / kGatherWarps;
          const int items = nh * nf;
          constexpr int kBatch = 8;
          for (int j0 = 0; j0 < items; j0 += 32 * kBatch) {
            double hv[kBatch];
#pragma unroll
            for (int i = 0; i < kBatch; i++) {
              const int j = j0 + lane + 32 * i;
              if (j < items) {
                const int h = j / nf, f = gw + kGatherWarps * (j - h * nf);
                hv[i] = ld_cg((f < 7 ? a.sg[f] : a.s[from][f - 7]) + rec[kRecHalo + h]);
              }
            }
#pragma unroll
            for (int i = 0; i < kBatch; i++) {
              const int j = j0 + lane + 32 * i;
              if (j < items) {
                const int h = j / nf, f = gw + kGatherWarps * (j - h * nf);
                st.hf[f][h] = hv[i];
              }
            }
          }
          if (gw == kGatherWarps - 1)
            for (int h = lane; h < nh; h += 32) st.hmeta[h] = a.meta[rec[kRecHalo + h]];
          mbar_arrive(&S.sfull[s]);
        }
        if (gw == 0 && lane == 0) trace_stamp(a, issued, 7);
      }
      // the record's generic reads come before its async-proxy refill
      fence_proxy_async();
      stage_sync();  // handshake 2
      if (pw == 0) {
        if (lane == 0) trace_stamp(a, issued, 0);
        const int qr = q + kRecRing;
        if (lane == 0 && qr < nq) {
          mbar_arrive_expect_tx(&S.rec_full[r], kRecBytes);
          bulk_g2s(S.rec[r], a.tile_rec + (size_t)(T0 + (kMulti ? qr % n : qr)) * kRecInts, kRecBytes,
                   &S.rec_full[r]);
        }
        if (a.prefetch > 0 && !multi) {
          const int tp = t + a.prefetch;
          if (tp < T1 && lane < 15) {
            // what the stage load of a later tile copies: its constant block,
            // the owned ranges of the 12 stresses, u and v
            const int po = a.tile_meta[8 * tp], pc = a.tile_meta[8 * tp + 1];
            const uint32_t pb = (uint32_t)((pc + 3) & ~3) * 8u;
            if (lane == 0)
              bulk_prefetch_l2(a.cblk + (size_t)tp * kBlk, (uint32_t)(kBlk * 8u));
            else if (lane <= 12)
              bulk_prefetch_l2(a.s[from][lane - 1] + po, pb);
            else
              bulk_prefetch_l2((lane == 13 ? u_in : v_in) + po, pb);
          }
        }
        if (multi) {
          if (lane == 0) publish(q);
          // the counters of the next step's dependencies, read ahead
          const int q1 = q + 1;
          if (q1 < nq && q1 / n > 0) {
            const int t1 = T0 + q1 % n, d = a.dep_off[t1] + lane;
            seen = d < a.dep_off[t1 + 1] ? ld_relaxed(a.epoch + a.dep_idx[d]) : 0u;
          }
        }
      }
      issued++;
    }
    if (pw == 0) {
      if (ok && lane == 0) {
        // the stepu parts of the last steps
        for (; nu < issued; nu++) {
          if (!mbar_wait(&S.uempty, (uint32_t)(nu - 1) & 1, a.err, 9)) break;
          issue_stepu(nu);
        }
      }
      if (lane == 0 && nu > 0) mbar_wait(&S.ufull, (uint32_t)(nu - 1) & 1, a.err, 10);
      if (multi && lane == 0) {
        // the last steps' counters (a later launch zeroes them anyway)
        const unsigned long long t0 = global_ns();
        while (ok && pub < issued && global_ns() - t0 < kWaitNs) publish(issued);
      }
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
        for (int k = issued; k < issued + kRecRing && k < nq; k++)
          mbar_wait(&S.rec_full[k % kRecRing], (uint32_t)(k / kRecRing) & 1, a.err, 7);
      }
    }
    __syncwarp();
    return;
  }

  // ========================= consumers ===================================
  // Per step one block barrier: after stress, when the tile's str table is
  // complete.  Stepu then runs warp by warp and each warp goes straight on to
  // the next step's stress, so one warp's stepu overlaps the others' stress.
  // Stepu of step q reads the tables of steps q and q-1 while stress of step
  // q+1 writes the third; the table it writes last held step q-2, whose
  // readers (stepu of q-2 and q-1) every warp has finished before any passes
  // the barrier of step q.  (The first tile of a run never reads the previous
  // table, so nothing crosses from one subcycle to the next there.)  The
  // stepu slot is released by one arrival per warp.  A wait that ran out
  // anywhere is OR-reduced at the barrier, so all consumers leave the loop
  // together.
  const int c = tid;  // compute-set index: owned c < cnt, halo cnt + h
  const int lane = tid & 31;
  bool fail = false;
  // Consumers write the ping-pong set the previous subcycle read: only after
  // it has completed (their first tile cannot land before that anyway).
  griddep_wait();


  // What stepu of a tile needs from its stress part, kept by the owned
  // thread so that the slot can be released after stress.
  struct Carry {
    uint32_t m = 0;
    uint32_t sg = 0;  // sign bits of uinit (bit 0) and vinit (bit 1)
    double uold = 0.0, vold = 0.0;
    int off = 0, cnt = 0;
  };

  // ---------------- stress of step q ---------------------------------------
  auto stress_tile = [&](int q) -> Carry {
    Carry cy;
    const int s = q % kSSlots;
    const int b = q % 3;
    const int sub = kMulti ? q / n : 0;
    const int to = (sub & 1) ^ 1;
    const bool wlast = kMulti ? (a.last && sub == a.nsub - 1) : kLast;
    const bool have = mbar_wait(&S.sfull[s], (uint32_t)(q / kSSlots) & 1, a.err, 1);
    fail |= !have;
    if (tid == 0) trace_stamp(a, q, 1);
    const SSlot &st = S.ss[s];
    if (have) {
      cy.off = st.hdr[0];
      cy.cnt = st.hdr[1];
      const int nh = st.hdr[2];
      const bool own = c < cy.cnt;
      const int h = c - cy.cnt;
      if (own || h < nh) {
        uint32_t m, lc;
        if (own) {
          const unsigned long long ml = (unsigned long long)__double_as_longlong(st.cs[7][c]);
          m = (uint32_t)ml;
          lc = (uint32_t)(ml >> 32);
          cy.m = m;
          cy.sg = lc >> 30;
          cy.uold = st.u[c];
          cy.vold = st.v[c];
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
            for (int k = 0; k < 12; k++) a.s[to][k][cy.off + c] = s12[k];
          }
        }
#pragma unroll
        for (int k = 0; k < 8; k++) S.str[b][k][c] = out[k];
        if (wlast && own) {
#pragma unroll
          for (int k = 0; k < 8; k++) a.str_out[k][cy.off + c] = out[k];
        }
      }
    }
    return cy;
  };

  // ---------------- stepu of step q, owned points ------------------------
  auto stepu_tile = [&](int q, const Carry &cy) {
    const int b = q % 3;
    const int bp = (q + 2) % 3;  // the previous tile's table
    const int sub = kMulti ? q / n : 0;
    const int to = (sub & 1) ^ 1;
    const bool wlast = kMulti ? (a.last && sub == a.nsub - 1) : kLast;
    const bool hu = mbar_wait(&S.ufull, (uint32_t)q & 1, a.err, 11);
    fail |= !hu;
    const bool act = hu && c < cy.cnt && !((cy.m >> 30) & kSkipU);
    // the 13 stepu inputs into registers first, so that the stepu slot is
    // released before the arithmetic: the bulk warp then issues the next
    // tile's stepu part and, behind it, the stress part after next a whole
    // stepu earlier.  (In a launch of several subcycles the release also
    // tells the bulk warp that the tile's velocities are stored, which it
    // publishes to other CTAs: there it stays after the stores.)
    StepuIn in;
    if (act) {
      const USlot &us = S.us;
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
      if (cpt) {
        // Tbu is +0; revp == 0, so revp*uinit is a zero with uinit's sign
        in.Tbu = 0.0;
        in.uinit = (cy.sg & 1u) ? -1.0 : 1.0;
        in.vinit = (cy.sg & 2u) ? -1.0 : 1.0;
      } else {
        in.Tbu = us.cu[10][c];
        in.uinit = us.cu[11][c];
        in.vinit = us.cu[12][c];
      }
    }
    if (!kMulti) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.uempty);  // this warp is done with the stepu slot
    }
    if (act) {
      const uint32_t m = cy.m;
      const double(&str)[8][kStrRow] = S.str[b];
      // a neighbour's str: own table, or the previous tile's (kStrPrev)
      const uint32_t vnw = m & kLnbMask, vsw = (m >> kLnbBits) & kLnbMask;
      const uint32_t vsse = (m >> (2 * kLnbBits)) & kLnbMask;
      const double(&tnw)[8][kStrRow] = (vnw & kStrPrev) ? S.str[bp] : S.str[b];
      const double(&tsw)[8][kStrRow] = (vsw & kStrPrev) ? S.str[bp] : S.str[b];
      const double(&tsse)[8][kStrRow] = (vsse & kStrPrev) ? S.str[bp] : S.str[b];
      const int lnw = vnw & (kStrPrev - 1), lsw = vsw & (kStrPrev - 1);
      const int lsse = vsse & (kStrPrev - 1);
      in.uold = cy.uold;
      in.vold = cy.vold;
      in.s1 = str[0][c];
      in.s2nw = tnw[1][lnw];
      in.s3sse = tsse[2][lsse];
      in.s4sw = tsw[3][lsw];
      in.s5 = str[4][c];
      in.s6sse = tsse[5][lsse];
      in.s7nw = tnw[6][lnw];
      in.s8sw = tsw[7][lsw];
      const StepuOut o = stepu_point(in, p);
      double *u_out = kMulti && a.uv_step ? a.u[0] + (size_t)(sub + 1) * a.uv_step : a.u[to];
      double *v_out = kMulti && a.uv_step ? a.v[0] + (size_t)(sub + 1) * a.uv_step : a.v[to];
      u_out[cy.off + c] = o.u;
      v_out[cy.off + c] = o.v;
      if (wlast) {
        a.strintx[cy.off + c] = o.strintx;
        a.strinty[cy.off + c] = o.strinty;
        a.Cb[cy.off + c] = o.Cb;
      }
    }
    if (kMulti) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.uempty);
    }
    if (tid == 0) trace_stamp(a, q, 5);
  };

  // the barrier after stress of step q: its str table is complete and its
  // stress slot free again
  auto stress_done = [&](int q) -> bool {
    const bool stop = consumer_sync_or(fail);
    if (tid == 0) {
      trace_stamp(a, q, 2);
      mbar_arrive(&S.sempty[q % kSSlots]);
    }
    return stop;
  };

  Carry cur = stress_tile(0);
  if (stress_done(0)) return;
  for (int q = 0; q < nq; q++) {
    stepu_tile(q, cur);
    if (q + 1 >= nq) break;
    const Carry nxt = stress_tile(q + 1);
    if (stress_done(q + 1)) break;
    cur = nxt;
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

// The same for the dependency wait of a multi-subcycle launch: one thread
// waits on a counter that nothing raises.
constexpr int kDepProbeCode = 14;

__global__ void k_dep_probe(int *err, const unsigned *counter, unsigned long long limit_ns) {
  if (threadIdx.x == 0) wait_counter(counter, 1u, err, kDepProbeCode, limit_ns);
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
    case 9: return "the stepu-part warp waited for the stepu slot";
    case 10: return "the stepu-part warp waited for its last copy";
    case 11: return "a consumer waited for a tile's stepu inputs";
    case 13: return "the producer waited for neighbouring tiles to finish a subcycle";
    case kProbeCode: return "the wait probe (evp1d_debug_wait_timeout)";
    case kDepProbeCode: return "the dependency-wait probe (evp1d_debug_dep_wait_timeout)";
    default: return "unknown";
  }
}

cudaError_t tma_binary_version(int *version) {
  cudaFuncAttributes at;
  const cudaError_t e = cudaFuncGetAttributes(&at, k_tma<false, true, false>);
  if (e == cudaSuccess) *version = at.binaryVersion;
  return e;
}

void launch_wait_probe(int *err, unsigned long long limit_ns, cudaStream_t st) {
  k_wait_probe<<<1, 32, 0, st>>>(err, limit_ns);
}

void launch_dep_probe(int *err, const unsigned *counter, unsigned long long limit_ns,
                      cudaStream_t st) {
  k_dep_probe<<<1, 32, 0, st>>>(err, counter, limit_ns);
}

using TmaKernel = void (*)(TmaArgs, Params);
constexpr int kTmaKernels = 6;
const TmaKernel kTmaAll[kTmaKernels] = {
    k_tma<false, false, false>, k_tma<true, false, false>, k_tma<false, true, false>,
    k_tma<true, true, false>,   k_tma<false, false, true>, k_tma<false, true, true>};

int tma_prepare(int device) {
  const int bytes = (int)smem_bytes();
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < kTmaKernels && e == cudaSuccess; i++)
    e = cudaFuncSetAttribute(kTmaAll[i], cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  (void)device;
  return e == cudaSuccess ? 0 : (int)e;
}

bool tma_can_persist(int device, int nruns) {
  int coop = 0, sms = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tma<false, true, true>, kThreads,
                                                    smem_bytes()) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return coop != 0 && nruns <= sms * per_sm;
}

cudaError_t launch_tma(const TmaArgs &given, const Params &p, cudaStream_t st) {
  if (given.ntiles <= 0 || given.nruns <= 0 || given.nsub <= 0) return cudaSuccess;
  TmaArgs a = given;
  // the short stepu part replaces revp*uinit by a signed zero: revp == 0 only
  a.compact = given.compact && given.cflags && p.revp == 0.0;
  const bool std = std_params(p);
  if (a.nsub > 1 && a.epoch) {
    // CTAs wait on one another: all of them resident at once
    TmaKernel k = std ? k_tma<false, true, true> : k_tma<false, false, true>;
    TmaArgs aa = a;
    Params pp = p;
    void *args[] = {&aa, &pp};
    return cudaLaunchCooperativeKernel((const void *)k, dim3(a.nruns), dim3(kThreads), args,
                                       smem_bytes(), st);
  }
  if (a.nsub != 1) return cudaErrorInvalidValue;  // several subcycles need the counters
  TmaKernel k = a.last ? (std ? k_tma<true, true, false> : k_tma<true, false, false>)
                       : (std ? k_tma<false, true, false> : k_tma<false, false, false>);
  if (a.pdl) {
    // a programmatic dependent of the previous launch on the stream, which
    // must be the previous subcycle's k_tma (the caller's guarantee)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(a.nruns);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem_bytes();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, a, p);
  }
  k<<<a.nruns, kThreads, smem_bytes(), st>>>(a, p);
  return cudaGetLastError();
}

}  // namespace evp
