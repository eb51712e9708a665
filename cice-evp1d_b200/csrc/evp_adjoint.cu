// evp_adjoint.cu -- reverse-mode gradients of the EVP subcycle loop.
//
// Forward (recording) pass: the ordinary fused subcycles, saving either
//  - every subcycle's velocities (a full velocity tape, when it fits the
//    device memory budget), or
//  - (u, v, 12 stresses) every `interval` subcycles (checkpoints).
// Reverse sweep, subcycle n = ndte-1 .. 0, in the solver's slot order:
//  - checkpoint mode first recomputes the velocities of one segment from its
//    checkpoint with the forward kernel into a segment tape;
//  - k_adj_stepu: per U point, the velocity adjoint lam_u(n+1) is completed
//    by gathering the stress kernel's corner contributions, then stepu is
//    reversed (src/bench_v2b.F90:509-544): lam_u(n) through stepu, the
//    adjoint of strintx/strinty scaled by uarear, and the forcex, forcey and
//    Cw gradients;
//  - k_adj_stress: per T point, the str adjoints are gathered from the U
//    points that read them (nw/sse/sw transposed), str_combine, the corner
//    relaxations and the strain rates are reversed (src/bench_v2b.F90:
//    137-310, 363-437); the stress adjoint is updated in place and the
//    strength gradient accumulated.
// Every neighbour access of the reverse sweep is a gather through transposed
// neighbour lists built once per handle, so the sweep uses no atomics and is
// deterministic.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "evp1d.h"
#include "evp_adjoint_math.cuh"
#include "evp_handle.h"
#include "evp_internal.h"

namespace evp {

namespace {

constexpr int kThreads = 256;

#define ADJ_TRY(x)                                                         \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess)                                                 \
      return error(e_ == cudaErrorMemoryAllocation ? EVP1D_ERR_NOMEM       \
                                                   : EVP1D_ERR_CUDA,       \
                   "%s: %s", #x, cudaGetErrorString(e_));                  \
  } while (0)

#define ADJ_CHECK(x)                \
  do {                              \
    int rc_ = (x);                  \
    if (rc_ != EVP1D_OK) return rc_; \
  } while (0)

// Transposed neighbour lists (CSR over slots).
enum {
  kTrNw = 0,   // U points x with nw(x) = w   (they read str2, str7 at w)
  kTrSse = 1,  // U points x with sse(x) = w  (str3, str6)
  kTrSw = 2,   // U points x with sw(x) = w   (str4, str8)
  kTrEe = 3,   // T points w with ee(w) = x   (they read u, v at x as "ee")
  kTrNe = 4,   // T points w with ne(w) = x
  kTrSe = 5,   // T points w with se(w) = x
  kNumTr = 6
};
enum { kGStrength, kGCw, kGForcex, kGForcey, kGUinit, kGVinit, kNumGrad };

struct AdjArgs {
  int nslots = 0;
  const uint8_t *flags = nullptr;
  const int32_t *ee = nullptr, *ne = nullptr, *se = nullptr;
  const int32_t *tr_off[kNumTr] = {}, *tr_idx[kNumTr] = {};
  // when no list has more than one entry (grid-shaped problems): the entry or
  // -1 per slot, read instead of the CSR lists
  const int32_t *tr_one[kNumTr] = {};
  const double *dxT = nullptr, *dyT = nullptr, *HTE = nullptr, *HTN = nullptr;
  const double *HTEm1 = nullptr, *HTNm1 = nullptr, *uarear = nullptr;
  const double *strength = nullptr, *kvrel = nullptr, *aiu = nullptr;
  const double *uocn = nullptr, *vocn = nullptr, *waterx = nullptr, *watery = nullptr;
  const double *umassdti = nullptr, *fm = nullptr, *Tbu = nullptr;
  double *Pu = nullptr, *Pv = nullptr;  // lam of u, v through stepu alone
  double *Lx = nullptr, *Ly = nullptr;  // uarear * lam of strintx, strinty
  double *C8[8] = {};                   // lam of the 8 corner velocities of a T point
  double *LS[12] = {};                  // lam of the 12 stresses
  double *g[kNumGrad] = {};
};

// lam of u(n+1), v(n+1) at x: stepu's own part plus the stress corners that
// read the velocity at x (as cc of x, and as ee/ne/se of other T points).
// With one entry per transposed list (kOne) each U point has at most one
// such T point per role, and k_adj_stress stores that corner's share at the
// U point's own slot (C8[2..7] indexed by x; slots no T point writes keep the
// zeros of the seed): the sum reads x's slots straight, with no index.
template <bool kOne>
__device__ __forceinline__ void velocity_lam(const AdjArgs &a, int x, double &lu,
                                             double &lv) {
  lu = a.Pu[x] + a.C8[0][x];
  lv = a.Pv[x] + a.C8[1][x];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (kOne) {
      lu += a.C8[2 + 2 * k][x];
      lv += a.C8[3 + 2 * k][x];
    } else {
      const int32_t *off = a.tr_off[kTrEe + k], *idx = a.tr_idx[kTrEe + k];
      const int b = off[x], e = off[x + 1];
      for (int q = b; q < e; q++) {
        const int w = idx[q];
        lu += a.C8[2 + 2 * k][w];
        lv += a.C8[3 + 2 * k][w];
      }
    }
  }
}

// Sum of Lx and Ly over the U points of transposed list t at slot w.
template <bool kOne>
__device__ __forceinline__ void str_lam(const AdjArgs &a, int t, int w, double &sx,
                                        double &sy) {
  sx = 0.0;
  sy = 0.0;
  if (kOne) {
    const int x = a.tr_one[t][w];
    if (x >= 0) {
      sx = a.Lx[x];
      sy = a.Ly[x];
    }
  } else {
    const int32_t *off = a.tr_off[t], *idx = a.tr_idx[t];
    for (int q = off[w]; q < off[w + 1]; q++) {
      sx += a.Lx[idx[q]];
      sy += a.Ly[idx[q]];
    }
  }
}

template <bool kOne>
__global__ void __launch_bounds__(kThreads, 3)  // 80 registers: 24 warps per SM, no spills
k_adj_stepu(AdjArgs a, Params p, const double *__restrict__ u0, const double *__restrict__ v0,
            const double *__restrict__ u1, const double *__restrict__ v1) {
  // launched as a programmatic dependent: the previous kernel's results
  // (and its reads of what this one writes) are complete after the wait
  griddep_launch_dependents();
  griddep_wait();
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < a.nslots;
       x += gridDim.x * blockDim.x) {
    // Every input is loaded before the skip test (all arrays hold nslots
    // entries), so the loads go out in one round instead of two.
    double lu, lv;
    velocity_lam<kOne>(a, x, lu, lv);
    const bool skip = a.flags[x] & kSkipU;
    StepuAdjIn in;
    in.uold = u0[x];
    in.vold = v0[x];
    in.unew = u1[x];
    in.vnew = v1[x];
    in.lun = lu;
    in.lvn = lv;
    in.kvrel = a.kvrel[x];
    in.aiXrhow = a.aiu[x] * p.rhow;
    in.uocn = a.uocn[x];
    in.vocn = a.vocn[x];
    in.waterx = a.waterx[x];
    in.watery = a.watery[x];
    in.umassdti = a.umassdti[x];
    in.fm = a.fm[x];
    in.Tbu = a.Tbu[x];
    const double ar = a.uarear[x];
    const double gfx = a.g[kGForcex][x], gfy = a.g[kGForcey][x], gcw = a.g[kGCw][x];
    // a skipped point (u(n+1) = u(n) there) passes lam on unchanged and
    // takes no gradient; selects, not branches, keep the loads above
    const StepuAdjOut o = stepu_adjoint(in, p);
    a.Pu[x] = skip ? lu : o.luold;
    a.Pv[x] = skip ? lv : o.lvold;
    a.Lx[x] = skip ? 0.0 : ar * o.lcc1;
    a.Ly[x] = skip ? 0.0 : ar * o.lcc2;
    a.g[kGForcex][x] = skip ? gfx : gfx + o.lcc1;
    a.g[kGForcey][x] = skip ? gfy : gfy + o.lcc2;
    a.g[kGCw][x] = skip ? gcw : gcw + o.gCw;
    if (p.revp != 0.0 && !skip) {
      a.g[kGUinit][x] += o.luinit;
      a.g[kGVinit][x] += o.lvinit;
    }
  }
}

// The 8 corner velocity adjoints of T point w: cc at w's slot; ee, ne, se at
// w's slot (read back through the transposed lists), or with kOne at the
// slots of those U points (velocity_lam), halo slots having no U point.
template <bool kOne>
__device__ __forceinline__ void store_corners(const AdjArgs &a, int w, int iee, int ine, int ise,
                                              const double (&lc)[8]) {
  a.C8[0][w] = lc[0];
  a.C8[1][w] = lc[1];
  if (kOne) {
    const int t[3] = {iee, ine, ise};
#pragma unroll
    for (int k = 0; k < 3; k++) {
      if (t[k] < a.nslots) {
        a.C8[2 + 2 * k][t[k]] = lc[2 + 2 * k];
        a.C8[3 + 2 * k][t[k]] = lc[3 + 2 * k];
      }
    }
  } else {
#pragma unroll
    for (int k = 2; k < 8; k++) a.C8[k][w] = lc[k];
  }
}

template <bool kOne>
__global__ void __launch_bounds__(kThreads, 2)
k_adj_stress(AdjArgs a, Params p, const double *__restrict__ u, const double *__restrict__ v) {
  griddep_launch_dependents();
  griddep_wait();
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < a.nslots;
       w += gridDim.x * blockDim.x) {
    const int iee = a.ee[w], ine = a.ne[w], ise = a.se[w];
    if (a.flags[w] & kSkipT) {  // stresses unchanged, str not written
      double zero[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      store_corners<kOne>(a, w, iee, ine, ise, zero);
      continue;
    }
    double lo[8];
    lo[0] = a.Lx[w];
    lo[4] = a.Ly[w];
    str_lam<kOne>(a, kTrNw, w, lo[1], lo[6]);
    str_lam<kOne>(a, kTrSse, w, lo[2], lo[5]);
    str_lam<kOne>(a, kTrSw, w, lo[3], lo[7]);
    double ls[12];
#pragma unroll
    for (int k = 0; k < 12; k++) ls[k] = a.LS[k][w];
    Corners c;
    c.ucc = u[w];
    c.vcc = v[w];
    c.uee = u[iee];
    c.vee = v[iee];
    c.une = u[ine];
    c.vne = v[ine];
    c.use = u[ise];
    c.vse = v[ise];
    const Geom g = make_geom_fw(a.dxT[w], a.dyT[w], a.HTE[w], a.HTN[w], a.HTEm1[w],
                             a.HTNm1[w], p.deltaminEVP);
    double lc[8], lstr;
    stress_adjoint(c, g, a.strength[w], p, lo, ls, lc, lstr);
#pragma unroll
    for (int k = 0; k < 12; k++) a.LS[k][w] = ls[k];
    store_corners<kOne>(a, w, iee, ine, ise, lc);
    a.g[kGStrength][w] += lstr;
  }
}

// lam of the velocities at call start; fold_init adds the uvel_init part
// when uvel_init was the call-start velocity.
template <bool kOne>
__global__ void __launch_bounds__(kThreads) k_adj_final(AdjArgs a, int fold_init) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < a.nslots;
       x += gridDim.x * blockDim.x) {
    double lu, lv;
    velocity_lam<kOne>(a, x, lu, lv);
    if (fold_init) {
      lu += a.g[kGUinit][x];
      lv += a.g[kGVinit][x];
    }
    a.Pu[x] = lu;
    a.Pv[x] = lv;
  }
}

// The forward kernels write u, v only at the slots they update (U points that
// are not skipU); the ping-pong buffers keep the constant rest.  Tape entries
// get that constant part -- skipU and padding slots [0, nslots) and halo
// slots [nslots, nuv) -- from su (blockIdx.y 0) and sv (1), for entries
// 1..count-1 of a tape whose entries are `entry_step` doubles apart, v at
// v_off after u.  One thread per slot: a slot the kernels update returns at
// once, a constant one reads its value once and stores it into every entry.
__global__ void k_fill_constant(double *tape, size_t entry_step, size_t v_off, int nslots,
                                int nuv, int count, const double *su, const double *sv,
                                const uint8_t *flags) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nuv || (j < nslots && !(flags[j] & kSkipU))) return;
  const double x = (blockIdx.y ? sv : su)[j];
  double *t = tape + (blockIdx.y ? v_off : 0) + j;
  for (int e = 1; e < count; e++) t[(size_t)e * entry_step] = x;
}

// One checkpoint's state: u, v (nuv doubles each) and the 12 stresses
// (nslots each), array blockIdx.y, copied in one launch.
struct StateCopy {
  const double *src[14];
  double *dst[14];
};

__global__ void k_copy_state(StateCopy c, int nuv, int nslots) {
  const int q = blockIdx.y;
  const int n = q < 2 ? nuv : nslots;
  const double *__restrict__ src = c.src[q];
  double *__restrict__ dst = c.dst[q];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = src[i];
}

int blocks_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > 148LL * 64) b = 148LL * 64;
  return (int)b;
}

// element counts rounded up to whole 256-byte lines
size_t pad256(size_t doubles) { return (doubles + 31) & ~size_t(31); }
size_t pad_ints(size_t n) { return (n + 63) & ~size_t(63); }

}  // namespace

struct AdjointState {
  int device = 0;
  // static part: transposed lists and work arrays (allocated once)
  void *arena = nullptr;
  size_t arena_bytes = 0;
  int32_t *tr_off[kNumTr] = {}, *tr_idx[kNumTr] = {};
  int32_t *tr_one[kNumTr] = {};
  bool one = false;  // every transposed list has at most one entry
  double *Pu = nullptr, *Pv = nullptr, *Lx = nullptr, *Ly = nullptr;
  double *C8[8] = {}, *LS[12] = {}, *g[kNumGrad] = {};
  double *spp[2][12] = {};  // stress ping-pong of the segment recompute
  // recording
  void *store = nullptr;
  size_t store_bytes = 0;
  size_t stride = 0;    // doubles per velocity tape entry (nuv, padded)
  size_t sstride = 0;   // doubles per stress array of a checkpoint (nslots, padded)
  // Subcycles [0, n_cp) are covered by checkpoints every `interval`
  // subcycles (nck of them) and recomputed segment by segment in the sweep;
  // subcycles [n_cp, ndte) keep every velocity state on the tape.
  double *ck = nullptr;    // nck checkpoints of u, v (stride each), 12 stresses
  double *tape = nullptr;  // tape entries: u then v, 2*stride doubles each
  int tape_entries = 0;
  // Tape entries [0, ndte - n_cp] hold the taped tail (when n_cp < ndte);
  // the sweep recomputes a checkpointed segment into interval + 1 entries
  // from seg_base on, after the tail, so the tail survives for later sweeps.
  int seg_base = 0;
  bool valid = false, uinit_explicit = false, seeded = false;
  int ndte = 0, interval = 0, nck = 0, n_cp = 0;
  long long budget = 0;  // bytes for checkpoints and tape (0: 80% of free memory)
  long long launches = 0;
};

void adjoint_release(AdjointState *a) {
  if (!a) return;
  cudaSetDevice(a->device);
  if (a->store) cudaFree(a->store);
  if (a->arena) cudaFree(a->arena);
  delete a;
}

void adjoint_invalidate(AdjointState *a) {
  if (a) {
    a->valid = false;
    a->seeded = false;
  }
}

namespace {

// Transposed neighbour lists and work arrays, built on first use.
int ensure_static(evp1d_t *h) {
  if (h->adj && h->adj->arena) return EVP1D_OK;
  DeviceProblem &d = h->d;
  if (!h->adj) h->adj = new AdjointState();
  AdjointState &A = *h->adj;
  A.device = d.device;
  const int S = d.nslots;
  cudaStream_t st = d.stream;
  // neighbours and slot -> point map from the device
  std::vector<int32_t> nb((size_t)6 * S), pos((size_t)S);
  for (int k = 0; k < 6; k++)
    ADJ_TRY(cudaMemcpyAsync(nb.data() + (size_t)k * S, d.nb[k], sizeof(int32_t) * S,
                            cudaMemcpyDeviceToHost, st));
  ADJ_TRY(cudaMemcpyAsync(pos.data(), d.point_of_slot, sizeof(int32_t) * S,
                          cudaMemcpyDeviceToHost, st));
  ADJ_TRY(cudaStreamSynchronize(st));
  auto nbk = [&](int k, int s) { return nb[(size_t)k * S + s]; };
  // (source neighbour vector, whether the edge is U->T or T->U) per list
  // nb order: 0 ee, 1 ne, 2 se, 3 nw, 4 sw, 5 sse
  const int src_nb[kNumTr] = {3, 5, 4, 0, 1, 2};
  std::vector<std::vector<int32_t>> off(kNumTr), idx(kNumTr);
  for (int t = 0; t < kNumTr; t++) {
    std::vector<int32_t> cnt((size_t)S + 1, 0);
    for (int s = 0; s < S; s++) {
      if (pos[s] < 0) continue;
      const int o = nbk(src_nb[t], s);
      if (o >= 0 && o < S && pos[o] >= 0) cnt[o + 1]++;
    }
    for (int s = 0; s < S; s++) cnt[s + 1] += cnt[s];
    off[t] = cnt;
    idx[t].assign((size_t)cnt[S], 0);
    std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
    for (int s = 0; s < S; s++) {  // ascending s: a fixed summation order
      if (pos[s] < 0) continue;
      const int o = nbk(src_nb[t], s);
      if (o >= 0 && o < S && pos[o] >= 0) idx[t][fill[o]++] = s;
    }
  }
  // direct form when no list has two entries
  bool one = true;
  for (int t = 0; t < kNumTr && one; t++)
    for (int w = 0; w < S; w++)
      if (off[t][w + 1] - off[t][w] > 1) {
        one = false;
        break;
      }
  std::vector<int32_t> direct;
  if (one) {
    direct.assign((size_t)kNumTr * S, -1);
    for (int t = 0; t < kNumTr; t++)
      for (int w = 0; w < S; w++)
        if (off[t][w + 1] > off[t][w]) direct[(size_t)t * S + w] = idx[t][off[t][w]];
  }
  A.one = one;
  // carve
  const size_t SD = pad256((size_t)S);
  size_t ints = one ? (size_t)kNumTr * pad_ints((size_t)S) : 0;
  for (int t = 0; t < kNumTr; t++) ints += pad_ints(off[t].size()) + pad_ints(idx[t].size() + 1);
  const size_t ndbl = SD * (4 + 8 + 12 + kNumGrad + 24);
  A.arena_bytes = ints * sizeof(int32_t) + ndbl * sizeof(double);
  ADJ_TRY(device_alloc(&A.arena, A.arena_bytes));
  double *pd = (double *)A.arena;
  auto take = [&]() {
    double *r = pd;
    pd += SD;
    return r;
  };
  A.Pu = take();
  A.Pv = take();
  A.Lx = take();
  A.Ly = take();
  for (int k = 0; k < 8; k++) A.C8[k] = take();
  for (int k = 0; k < 12; k++) A.LS[k] = take();
  for (int k = 0; k < kNumGrad; k++) A.g[k] = take();
  for (int b = 0; b < 2; b++)
    for (int k = 0; k < 12; k++) A.spp[b][k] = take();
  int32_t *pi = (int32_t *)pd;
  for (int t = 0; t < kNumTr; t++) {
    A.tr_off[t] = pi;
    pi += pad_ints(off[t].size());
    A.tr_idx[t] = pi;
    pi += pad_ints(idx[t].size() + 1);
    if (one) {
      A.tr_one[t] = pi;
      pi += pad_ints((size_t)S);
      ADJ_TRY(cudaMemcpyAsync(A.tr_one[t], direct.data() + (size_t)t * S, sizeof(int32_t) * S,
                              cudaMemcpyHostToDevice, st));
    }
    ADJ_TRY(cudaMemcpyAsync(A.tr_off[t], off[t].data(), sizeof(int32_t) * off[t].size(),
                            cudaMemcpyHostToDevice, st));
    if (!idx[t].empty())
      ADJ_TRY(cudaMemcpyAsync(A.tr_idx[t], idx[t].data(), sizeof(int32_t) * idx[t].size(),
                              cudaMemcpyHostToDevice, st));
  }
  ADJ_TRY(cudaStreamSynchronize(st));  // the host vectors go out of scope
  return EVP1D_OK;
}

AdjArgs adj_args(const evp1d_t *h) {
  const DeviceProblem &d = h->d;
  const AdjointState &A = *h->adj;
  AdjArgs a;
  a.nslots = d.nslots;
  a.flags = d.flags;
  a.ee = d.nb[0];
  a.ne = d.nb[1];
  a.se = d.nb[2];
  for (int t = 0; t < kNumTr; t++) {
    a.tr_off[t] = A.tr_off[t];
    a.tr_idx[t] = A.tr_idx[t];
    a.tr_one[t] = A.tr_one[t];
  }
  a.dxT = d.geo[kDxT];
  a.dyT = d.geo[kDyT];
  a.HTE = d.geo[kHTE];
  a.HTN = d.geo[kHTN];
  a.HTEm1 = d.geo[kHTEm1];
  a.HTNm1 = d.geo[kHTNm1];
  a.uarear = d.geo[kUarear];
  a.strength = d.dyn[kStrength];
  a.kvrel = d.dyn[kKvrel];
  a.aiu = d.dyn[kAiu];
  a.uocn = d.dyn[kUocn];
  a.vocn = d.dyn[kVocn];
  a.waterx = d.dyn[kWaterx];
  a.watery = d.dyn[kWatery];
  a.umassdti = d.dyn[kUmassdti];
  a.fm = d.dyn[kFm];
  a.Tbu = d.dyn[kTbu];
  a.Pu = A.Pu;
  a.Pv = A.Pv;
  a.Lx = A.Lx;
  a.Ly = A.Ly;
  for (int k = 0; k < 8; k++) a.C8[k] = A.C8[k];
  for (int k = 0; k < 12; k++) a.LS[k] = A.LS[k];
  for (int k = 0; k < kNumGrad; k++) a.g[k] = A.g[k];
  return a;
}

// One forward subcycle between explicit state buffers.  `after_sub`: the
// previous launch on the stream is the previous subcycle's (it may then start
// as its programmatic dependent).
void launch_state(evp1d_t *h, double *const s_in[12], double *const s_out[12],
                  const double *u_in, const double *v_in, double *u_out, double *v_out,
                  bool last, bool after_sub = false) {
  DeviceProblem &d = h->d;
  if (h->path == kPathTma) {
    TmaArgs a = problem_tma_args(d, 0);
    a.prefetch = h->prefetch;
    // one subcycle: set 0 is only read, set 1 only written
    for (int k = 0; k < 12; k++) {
      a.s[0][k] = s_in[k];
      a.s[1][k] = s_out[k];
    }
    a.u[0] = const_cast<double *>(u_in);
    a.v[0] = const_cast<double *>(v_in);
    a.u[1] = u_out;
    a.v[1] = v_out;
    a.nsub = 1;
    a.last = last;
    a.pdl = after_sub && h->pdl;
    launch_tma(a, h->p, d.stream);
  } else {
    FusedArgs a = problem_fused_args(d, 0);
    for (int k = 0; k < 12; k++) {
      a.s_in[k] = s_in[k];
      a.s_out[k] = s_out[k];
    }
    a.u_in = u_in;
    a.v_in = v_in;
    a.u_out = u_out;
    a.v_out = v_out;
    launch_fused(a, h->p, last, d.stream);
  }
}

// `len` forward subcycles from tape entry e0: the velocities of subcycle i go
// into entry e0 + i + 1, the stresses alternate between s0 and s1 (s0 holds
// the start).  One multi-subcycle launch where the handle runs those, else one
// launch per subcycle.
void launch_states(evp1d_t *h, double *const s0[12], double *const s1[12], double *tu0,
                   double *tv0, size_t entry_step, int len, bool last);

double *tape_u(AdjointState &A, int e) { return A.tape + (size_t)e * 2 * A.stride; }

void launch_states(evp1d_t *h, double *const s0[12], double *const s1[12], double *tu0,
                   double *tv0, size_t entry_step, int len, bool last) {
  DeviceProblem &d = h->d;
  if (len <= 0) return;
  if (h->path == kPathTma && h->persist && len > 1) {
    cudaMemsetAsync(d.epoch, 0, sizeof(unsigned) * (size_t)d.ntiles, d.stream);
    TmaArgs a = problem_tma_args(d, 0);
    for (int k = 0; k < 12; k++) {
      a.s[0][k] = s0[k];
      a.s[1][k] = s1[k];
    }
    a.u[0] = tu0;
    a.v[0] = tv0;
    a.uv_step = entry_step;
    a.nsub = len;
    a.last = last;
    a.epoch = d.epoch;
    launch_tma(a, h->p, d.stream);
    h->launches++;
    return;
  }
  for (int i = 0; i < len; i++) {
    const bool odd = i & 1;
    launch_state(h, odd ? s1 : s0, odd ? s0 : s1, tu0 + (size_t)i * entry_step,
                 tv0 + (size_t)i * entry_step, tu0 + (size_t)(i + 1) * entry_step,
                 tv0 + (size_t)(i + 1) * entry_step, last && i == len - 1, i > 0);
  }
  h->launches += len;
}

double *tape_v(AdjointState &A, int e) { return A.tape + (size_t)e * 2 * A.stride + A.stride; }
double *ck_u(AdjointState &A, int j) {
  return A.ck + (size_t)j * (2 * A.stride + 12 * A.sstride);
}
double *ck_v(AdjointState &A, int j) { return ck_u(A, j) + A.stride; }
double *ck_s(AdjointState &A, int j, int k) {
  return ck_u(A, j) + 2 * A.stride + (size_t)k * A.sstride;
}

int ensure_store(AdjointState &A, size_t bytes) {
  if (A.store && A.store_bytes >= bytes) return EVP1D_OK;
  if (A.store) cudaFree(A.store);
  A.store = nullptr;
  A.store_bytes = 0;
  ADJ_TRY(device_alloc(&A.store, bytes));
  A.store_bytes = bytes;
  return EVP1D_OK;
}

}  // namespace
}  // namespace evp

using namespace evp;

extern "C" {

int evp1d_record_subcycles(evp1d_t *h, int ndte, int interval) {
  evp::NvtxRange nvtx_range("evp1d_record_subcycles");
  if (!h) return error(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (ndte < 1) return error(EVP1D_ERR_INVALID_ARG, "ndte = %d < 1", ndte);
  if (!h->uploaded) return error(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  ADJ_TRY(cudaSetDevice(h->d.device));
  DeviceProblem &d = h->d;
  if (d.ntiles == 0) {  // nothing to differentiate
    if (!h->adj) h->adj = new AdjointState();
    h->adj->device = d.device;
    h->adj->valid = true;
    h->adj->ndte = ndte;
    h->adj->nck = 0;
    h->adj->n_cp = 0;
    h->adj->seeded = false;
    return EVP1D_OK;
  }
  ADJ_CHECK(ensure_static(h));
  AdjointState &A = *h->adj;
  A.valid = false;
  A.seeded = false;
  A.stride = pad256((size_t)d.nuv);
  A.sstride = pad256((size_t)d.nslots);
  const size_t entry = 2 * A.stride * sizeof(double);
  const size_t ckpt = (2 * A.stride + 12 * A.sstride) * sizeof(double);
  // split of the subcycles into a checkpointed head and a taped tail
  int k = 0, n_cp = 0;
  if (interval > 0) {
    // checkpoints every k subcycles, except for the last segment: the
    // recording tapes its velocities (the tape holds a segment anyway), so
    // the sweep reverses it without recomputing it
    k = std::min(interval, ndte);
    n_cp = k * ((ndte - 1) / k);
    if (n_cp == 0) k = 0;
  } else {
    size_t freeb = 0, totalb = 0;
    ADJ_TRY(cudaMemGetInfo(&freeb, &totalb));
    const double budget = A.budget > 0 ? (double)A.budget
                                       : 0.8 * (double)(freeb + A.store_bytes);
    if ((double)(ndte + 1) * (double)entry > budget) {
      // interval sqrt(ndte * checkpoint / tape entry) minimises the memory of
      // a checkpoints-only recording; the rest of the budget tapes the tail
      k = (int)std::ceil(std::sqrt((double)ndte * (double)ckpt / (double)entry));
      k = std::max(1, std::min(k, ndte));
      // the segment recompute needs k + 1 entries of its own; what is left
      // of the budget tapes the final subcycles (a tail of T needs T + 1)
      const double nck_max = std::ceil((double)ndte / k);
      const double left =
          std::floor((budget - nck_max * (double)ckpt) / (double)entry) - (double)(k + 1);
      const int tail = left >= 2.0 ? (int)std::min(left - 1.0, (double)ndte) : 0;
      n_cp = ndte - tail;
      if (n_cp == 0) k = 0;
    }
  }
  const int nck = n_cp > 0 ? (n_cp + k - 1) / k : 0;
  const int tail_entries = n_cp < ndte ? ndte - n_cp + 1 : 0;
  const int entries = tail_entries + (n_cp > 0 ? k + 1 : 0);
  ADJ_CHECK(ensure_store(A, (size_t)nck * ckpt + (size_t)entries * entry));
  A.ck = (double *)A.store;
  A.tape = A.ck + (size_t)nck * (ckpt / sizeof(double));
  A.tape_entries = entries;
  A.seg_base = tail_entries;
  A.interval = k;
  A.nck = nck;
  A.n_cp = n_cp;
  cudaStream_t st = d.stream;
  const int cur0 = d.cur;
  // the constant slots of every tape entry (entry 0 is copied whole each time)
  if (entries > 1) {
    const dim3 grid((unsigned)((d.nuv + kThreads - 1) / kThreads), 2);
    k_fill_constant<<<grid, kThreads, 0, st>>>(A.tape, 2 * A.stride, A.stride, d.nslots, d.nuv,
                                               entries, d.u[cur0], d.v[cur0], d.flags);
    h->launches++;
  }
  // checkpointed head: the ordinary subcycle loop with a copy of the state
  // at the start of every segment
  for (int j = 0; j < nck; j++) {
    const int c = d.cur;
    StateCopy cp;
    cp.src[0] = d.u[c];
    cp.src[1] = d.v[c];
    cp.dst[0] = ck_u(A, j);
    cp.dst[1] = ck_v(A, j);
    for (int q = 0; q < 12; q++) {
      cp.src[2 + q] = d.stress[c][q];
      cp.dst[2 + q] = ck_s(A, j, q);
    }
    k_copy_state<<<dim3(blocks_for(d.nuv), 14), kThreads, 0, st>>>(cp, d.nuv, d.nslots);
    h->launches++;
    ADJ_CHECK(evp1d_subcycles(h, std::min(k, n_cp - j * k)));
  }
  // taped tail: each subcycle writes its velocities into the next entry
  if (n_cp < ndte) {
    const int c = d.cur;
    ADJ_TRY(cudaMemcpyAsync(tape_u(A, 0), d.u[c], sizeof(double) * d.nuv,
                            cudaMemcpyDeviceToDevice, st));
    ADJ_TRY(cudaMemcpyAsync(tape_v(A, 0), d.v[c], sizeof(double) * d.nuv,
                            cudaMemcpyDeviceToDevice, st));
    launch_states(h, d.stress[c], d.stress[1 - c], tape_u(A, 0), tape_v(A, 0), 2 * A.stride,
                  ndte - n_cp, true);
    const int b = ((ndte - n_cp) & 1) ? 1 - c : c;
    // the final state back into the handle's buffers for evp1d_download
    ADJ_TRY(cudaMemcpyAsync(d.u[b], tape_u(A, ndte - n_cp), sizeof(double) * d.nslots,
                            cudaMemcpyDeviceToDevice, st));
    ADJ_TRY(cudaMemcpyAsync(d.v[b], tape_v(A, ndte - n_cp), sizeof(double) * d.nslots,
                            cudaMemcpyDeviceToDevice, st));
    d.cur = b;
  }
  ADJ_TRY(cudaGetLastError());
  A.ndte = ndte;
  A.uinit_explicit = h->uinit_explicit;
  A.valid = true;
  return EVP1D_OK;
}

int evp1d_run_checkpointed(evp1d_t *h, int ndte, const evp1d_fields *io, int interval) {
  ADJ_CHECK(evp1d_upload(h, io));
  ADJ_CHECK(evp1d_record_subcycles(h, ndte, interval));
  return evp1d_download(h, io);
}

int evp1d_adjoint_seed(evp1d_t *h, const double *lam_uvel, const double *lam_vvel,
                       const double *const *lam_stress) {
  evp::NvtxRange nvtx_range("evp1d_adjoint_seed");
  if (!h) return error(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (!h->adj || !h->adj->valid)
    return error(EVP1D_ERR_STATE, "no recorded forward: call evp1d_run_checkpointed first");
  DeviceProblem &d = h->d;
  AdjointState &A = *h->adj;
  if (d.ntiles == 0) {
    A.seeded = true;
    return EVP1D_OK;
  }
  if (!lam_uvel || !lam_vvel) return error(EVP1D_ERR_INVALID_ARG, "lam_uvel/lam_vvel are NULL");
  ADJ_TRY(cudaSetDevice(d.device));
  cudaStream_t st = d.stream;
  const size_t nv = (size_t)(d.navel > 0 ? d.navel : 1);
  const size_t bn = sizeof(double) * (size_t)d.na;
  PermBatch b;
  auto add = [&](const double *host, double *dst) -> int {
    double *slot = d.stage + (size_t)b.n * nv;
    ADJ_TRY(cudaMemcpyAsync(slot, host, bn, cudaMemcpyHostToDevice, st));
    b.src[b.n] = slot;
    b.dst[b.n] = dst;
    b.n++;
    return EVP1D_OK;
  };
  ADJ_CHECK(add(lam_uvel, A.Pu));
  ADJ_CHECK(add(lam_vvel, A.Pv));
  for (int k = 0; k < 12; k++) {
    if (lam_stress && lam_stress[k])
      ADJ_CHECK(add(lam_stress[k], A.LS[k]));
    else
      ADJ_TRY(cudaMemsetAsync(A.LS[k], 0, sizeof(double) * d.nslots, st));
  }
  launch_scatter(b, d.nslots, d.point_of_slot, st);
  for (int k = 0; k < 8; k++)
    ADJ_TRY(cudaMemsetAsync(A.C8[k], 0, sizeof(double) * d.nslots, st));
  for (int k = 0; k < kNumGrad; k++)
    ADJ_TRY(cudaMemsetAsync(A.g[k], 0, sizeof(double) * d.nslots, st));
  ADJ_TRY(cudaGetLastError());
  A.seeded = true;
  return EVP1D_OK;
}

int evp1d_adjoint_sweep(evp1d_t *h) {
  evp::NvtxRange nvtx_range("evp1d_adjoint_sweep");
  if (!h) return error(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (!h->adj || !h->adj->valid)
    return error(EVP1D_ERR_STATE, "no recorded forward: call evp1d_run_checkpointed first");
  AdjointState &A = *h->adj;
  if (!A.seeded) return error(EVP1D_ERR_STATE, "evp1d_adjoint_seed has not been called");
  DeviceProblem &d = h->d;
  A.seeded = false;  // the sweep consumes the seed
  if (d.ntiles == 0) return EVP1D_OK;
  ADJ_TRY(cudaSetDevice(d.device));
  cudaStream_t st = d.stream;
  const AdjArgs a = adj_args(h);
  const int grid = blocks_for(d.nslots);
  long long launches = 0;
  const bool one = A.one;
  // Both reverse kernels start as programmatic dependents of the kernel
  // before them (each waits for it before touching memory), so that a
  // launch's scheduling overlaps the previous one's last blocks.
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = h->pdl ? 1 : 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kThreads);
  cfg.stream = st;
  cfg.attrs = pdl;
  cfg.numAttrs = 1;
  cudaError_t le = cudaSuccess;
  auto keep = [&](cudaError_t e) {
    if (le == cudaSuccess) le = e;
  };
  auto reverse_step = [&](const double *u0, const double *v0, const double *u1,
                          const double *v1) {
    const Params &p = h->p;
    if (one) {
      keep(cudaLaunchKernelEx(&cfg, k_adj_stepu<true>, a, p, u0, v0, u1, v1));
      keep(cudaLaunchKernelEx(&cfg, k_adj_stress<true>, a, p, u0, v0));
    } else {
      keep(cudaLaunchKernelEx(&cfg, k_adj_stepu<false>, a, p, u0, v0, u1, v1));
      keep(cudaLaunchKernelEx(&cfg, k_adj_stress<false>, a, p, u0, v0));
    }
    launches += 2;
  };
  // taped tail
  for (int n = A.ndte - 1; n >= A.n_cp; n--) {
    const int e = n - A.n_cp;
    reverse_step(tape_u(A, e), tape_v(A, e), tape_u(A, e + 1), tape_v(A, e + 1));
  }
  // checkpointed head, one segment at a time from the last
  const int k = A.interval;
  for (int j = A.nck - 1; j >= 0; j--) {
    const int len = std::min(k, A.n_cp - j * k);
    const int e0 = A.seg_base;
    StateCopy cp;
    cp.src[0] = ck_u(A, j);
    cp.src[1] = ck_v(A, j);
    cp.dst[0] = tape_u(A, e0);
    cp.dst[1] = tape_v(A, e0);
    for (int q = 0; q < 12; q++) {
      cp.src[2 + q] = ck_s(A, j, q);
      cp.dst[2 + q] = A.spp[0][q];
    }
    k_copy_state<<<dim3(blocks_for(d.nuv), 14), kThreads, 0, st>>>(cp, d.nuv, d.nslots);
    launches++;
    // Recompute the segment's velocities from its checkpoint.  Its end state
    // is stored already -- the next checkpoint's u, v, or the taped tail's
    // first entry -- so the last subcycle is copied, not recomputed (the
    // forward is deterministic: the same bits).
    const bool end_stored = j + 1 < A.nck || A.n_cp < A.ndte;
    const int nrec = end_stored ? len - 1 : len;
    const long long before = h->launches;
    launch_states(h, A.spp[0], A.spp[1], tape_u(A, e0), tape_v(A, e0), 2 * A.stride, nrec,
                  false);
    launches += h->launches - before;
    h->launches = before;
    if (end_stored) {
      const double *eu = j + 1 < A.nck ? ck_u(A, j + 1) : tape_u(A, 0);
      const double *ev = j + 1 < A.nck ? ck_v(A, j + 1) : tape_v(A, 0);
      ADJ_TRY(cudaMemcpyAsync(tape_u(A, e0 + len), eu, sizeof(double) * d.nuv,
                              cudaMemcpyDeviceToDevice, st));
      ADJ_TRY(cudaMemcpyAsync(tape_v(A, e0 + len), ev, sizeof(double) * d.nuv,
                              cudaMemcpyDeviceToDevice, st));
    }
    for (int i = len - 1; i >= 0; i--)
      reverse_step(tape_u(A, e0 + i), tape_v(A, e0 + i), tape_u(A, e0 + i + 1),
                   tape_v(A, e0 + i + 1));
  }
  if (one)
    k_adj_final<true><<<grid, kThreads, 0, st>>>(a, A.uinit_explicit ? 0 : 1);
  else
    k_adj_final<false><<<grid, kThreads, 0, st>>>(a, A.uinit_explicit ? 0 : 1);
  launches++;
  ADJ_TRY(le);
  ADJ_TRY(cudaGetLastError());
  A.launches = launches;
  h->launches += launches;
  return EVP1D_OK;
}

int evp1d_adjoint_gradients(evp1d_t *h, const evp1d_grads *g) {
  evp::NvtxRange nvtx_range("evp1d_adjoint_gradients");
  if (!h || !g) return error(EVP1D_ERR_INVALID_ARG, "NULL argument");
  if (!h->adj || !h->adj->valid)
    return error(EVP1D_ERR_STATE, "no recorded forward: call evp1d_run_checkpointed first");
  DeviceProblem &d = h->d;
  AdjointState &A = *h->adj;
  ADJ_TRY(cudaSetDevice(d.device));
  cudaStream_t st = d.stream;
  if (d.na == 0) return EVP1D_OK;
  int code = 0;
  ADJ_CHECK(problem_take_error(&d, &code));
  if (code)
    return error(EVP1D_ERR_TIMEOUT,
                 "a bounded device-side wait ran out (code %d: %s); the gradients are not valid",
                 code, tma_wait_name(code));
  const size_t nv = (size_t)(d.navel > 0 ? d.navel : 1);
  const size_t bn = sizeof(double) * (size_t)d.na;
  struct Out {
    const double *src;
    double *host;
  };
  std::vector<Out> outs;
  auto want = [&](double *host, const double *src) {
    if (host) outs.push_back({src, host});
  };
  want(g->strength, A.g[kGStrength]);
  want(g->Cw, A.g[kGCw]);
  want(g->forcex, A.g[kGForcex]);
  want(g->forcey, A.g[kGForcey]);
  want(g->uvel, A.Pu);
  want(g->vvel, A.Pv);
  for (int k = 0; k < 12; k++) want(g->stress[k], A.LS[k]);
  if (A.uinit_explicit) {
    want(g->uvel_init, A.g[kGUinit]);
    want(g->vvel_init, A.g[kGVinit]);
  } else {
    if (g->uvel_init) memset(g->uvel_init, 0, bn);
    if (g->vvel_init) memset(g->vvel_init, 0, bn);
  }
  for (size_t o = 0; o < outs.size(); o += kMaxBatch) {
    PermBatch b;
    for (size_t q = o; q < outs.size() && b.n < kMaxBatch; q++) {
      b.src[b.n] = outs[q].src;
      b.dst[b.n] = d.stage + (size_t)b.n * nv;
      b.n++;
    }
    launch_gather(b, d.na, d.slot_of_point, st);
    for (int q = 0; q < b.n; q++)
      ADJ_TRY(cudaMemcpyAsync(outs[o + q].host, b.dst[q], bn, cudaMemcpyDeviceToHost, st));
    ADJ_TRY(cudaStreamSynchronize(st));
  }
  ADJ_TRY(cudaGetLastError());
  return EVP1D_OK;
}

int evp1d_adjoint(evp1d_t *h, const double *lam_uvel, const double *lam_vvel,
                  const double *const *lam_stress, const evp1d_grads *g) {
  ADJ_CHECK(evp1d_adjoint_seed(h, lam_uvel, lam_vvel, lam_stress));
  ADJ_CHECK(evp1d_adjoint_sweep(h));
  return evp1d_adjoint_gradients(h, g);
}

int evp1d_set_adjoint_budget(evp1d_t *h, long long bytes) {
  if (!h || bytes < 0) return error(EVP1D_ERR_INVALID_ARG, "bad arguments");
  if (!h->adj) {
    h->adj = new AdjointState();
    h->adj->device = h->d.device;
  }
  h->adj->budget = bytes;
  return EVP1D_OK;
}

int evp1d_adjoint_info(evp1d_t *h, long long info[8]) {
  if (!h || !info) return error(EVP1D_ERR_INVALID_ARG, "NULL argument");
  for (int k = 0; k < 8; k++) info[k] = 0;
  const AdjointState *A = h->adj;
  if (!A) return EVP1D_OK;
  info[0] = A->valid ? 1 : 0;
  info[1] = A->ndte - A->n_cp;
  info[2] = A->interval;
  info[3] = A->nck;
  info[4] = (long long)A->store_bytes;
  info[5] = (long long)A->arena_bytes;
  info[6] = (long long)h->d.arena_bytes;
  info[7] = A->launches;
  return EVP1D_OK;
}

}  // extern "C"
