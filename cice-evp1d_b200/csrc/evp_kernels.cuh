// evp_kernels.cuh -- device data layout and kernel launchers of the EVP-1D
// library (internal, not part of the C-ABI).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "evp_math.cuh"
#include "evp_tiles.h"

namespace evp {

// Programmatic dependent launch.  launch_dependents lets the next launch on
// the stream (when it was launched as a programmatic dependent) be scheduled
// once every CTA of this one has executed it or exited; its CTAs then take
// the room this launch's CTAs leave.  wait blocks until the previous launch
// has completed and its memory is visible (it returns at once in a launch
// that is not a programmatic dependent).
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ void griddep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Skip flags packed per slot: bit 0 = skipT, bit 1 = skipU.  Alignment
// padding slots carry both bits.
constexpr uint8_t kSkipT = 1;
constexpr uint8_t kSkipU = 2;

// Arrays of one in-place stress / stepu pass (the lindividual loops) over
// `na` slots.  Indices address u, v and str, which have `navel` entries.
struct DevState {
  int na = 0, navel = 0;
  const int32_t *ee = nullptr, *ne = nullptr, *se = nullptr;
  const int32_t *nw = nullptr, *sw = nullptr, *sse = nullptr;
  const uint8_t *flags = nullptr;
  const double *dxT = nullptr, *dyT = nullptr, *HTE = nullptr, *HTN = nullptr;
  const double *HTEm1 = nullptr, *HTNm1 = nullptr, *uarear = nullptr;
  const double *strength = nullptr, *Cw = nullptr, *aiu = nullptr;
  const double *uocn = nullptr, *vocn = nullptr, *waterx = nullptr;
  const double *watery = nullptr, *forcex = nullptr, *forcey = nullptr;
  const double *umassdti = nullptr, *fm = nullptr, *Tbu = nullptr;
  const double *uinit = nullptr, *vinit = nullptr;
  double *stress[12] = {};
  double *u = nullptr, *v = nullptr;
  double *str[8] = {};
  double *strintx = nullptr, *strinty = nullptr, *Cb = nullptr;
};

// One stress pass (src/bench_v2b.F90:62-312), in place.
void launch_stress(const DevState &s, const Params &p, cudaStream_t st);
// One stepu pass (src/bench_v2b.F90:444-549), in place.
void launch_stepu(const DevState &s, const Params &p, cudaStream_t st);

// One subcycle of the fused tile solver: stress on every tile's owned points
// and forward halo, str in shared memory, stepu on the owned points.  Reads
// the *_in state and writes the *_out state (ping-pong buffers).  CTA r works
// through the tiles of run r in order (a stepu str index may point into the
// previous tile's table).
struct FusedArgs {
  int ntiles = 0, nruns = 0;
  const int32_t *run_off = nullptr;  // [nruns + 1]
  const int32_t *tile_off = nullptr, *tile_cnt = nullptr;
  const int32_t *halo_off = nullptr, *halo_cnt = nullptr, *halo_idx = nullptr;
  const uint8_t *flags = nullptr;
  const int32_t *ee = nullptr, *ne = nullptr, *se = nullptr;
  const uint32_t *lnb = nullptr;
  const double *dxT = nullptr, *dyT = nullptr, *HTE = nullptr, *HTN = nullptr;
  const double *HTEm1 = nullptr, *HTNm1 = nullptr, *strength = nullptr;
  const double *kvrel = nullptr, *uocn = nullptr, *vocn = nullptr;
  const double *waterx = nullptr, *watery = nullptr, *forcex = nullptr;
  const double *forcey = nullptr, *umassdti = nullptr, *fm = nullptr;
  const double *uarear = nullptr, *Tbu = nullptr, *uinit = nullptr;
  const double *vinit = nullptr;
  const double *u_in = nullptr, *v_in = nullptr;
  double *u_out = nullptr, *v_out = nullptr;
  const double *s_in[12] = {};
  double *s_out[12] = {};
  // written on the last subcycle of a call only
  double *strintx = nullptr, *strinty = nullptr, *Cb = nullptr;
  double *str_out[8] = {};
};

void launch_fused(const FusedArgs &a, const Params &p, bool last,
                  cudaStream_t st);

// The same subcycle as a persistent producer/consumer kernel fed by TMA bulk
// copies (evp_kernels_tma.cu).  sf = 7 stress inputs (dxT, dyT, HTE, HTN,
// HTEm1, HTNm1, strength) then the 12 input stresses, read by the halo
// gathers and the stress copies; the 13 stepu inputs (kvrel, uocn, vocn,
// waterx, watery, forcex, forcey, umassdti, fm, uarear, Tbu, uinit, vinit)
// come from the constant blocks.
constexpr int kTmaStressFields = 19;
constexpr int kTmaStepuFields = 13;
// The stepu part without its last three fields (Tbu, uinit, vinit): enough
// when every Tbu of the call is +0 and every uinit, vinit is finite, and
// revp == 0 (TmaArgs::compact).  stepu then takes Tbu = +0, which is the
// value, and uinit = +-1 with uinit's sign (bits 62 and 63 of the packed
// word): revp*uinit is the same signed zero either way.
constexpr int kTmaStepuCompact = 10;
// Per-call constants of a tile in one contiguous block: kConstFields x
// kTileOwned doubles per tile, fields [0..5] dxT dyT HTE HTN HTEm1 HTNm1,
// [6] strength, [7] meta | lcor << 32 (the kConstStressFields that stress
// reads), then [8..20] the 13 stepu inputs in the uf order; unused slots
// hold 0.  Each of the two parts is one bulk copy.
constexpr int kConstStressFields = 8;
constexpr int kConstFields = kConstStressFields + kTmaStepuFields;
constexpr int kConstTileSlots = kTileOwned;
struct TmaArgs {
  int ntiles = 0, nruns = 0;
  const int32_t *run_off = nullptr;  // [nruns + 1]: CTA r's tiles
  const int32_t *tile_off = nullptr, *tile_cnt = nullptr;
  const int32_t *halo_off = nullptr, *halo_cnt = nullptr, *halo_idx = nullptr;
  const int32_t *uvx_off = nullptr, *uvx_cnt = nullptr, *uvx_idx = nullptr;
  const uint32_t *meta = nullptr, *lcor = nullptr;
  const uint32_t *halo_lcc = nullptr, *halo_lcor = nullptr;
  // per tile 8 int32: off, cnt, uvx_off, uvx_cnt, halo_off, halo_cnt, 0, 0
  const int32_t *tile_meta = nullptr;
  // per tile one producer record of kRecInts int32 (evp_tiles.h)
  const int32_t *tile_rec = nullptr;
  // dxT, dyT, HTE, HTN, HTEm1, HTNm1, strength (the halo's static gathers)
  const double *sg[7] = {};
  const double *cblk = nullptr;  // constant blocks, kConstFields x kTileOwned per tile
  // the ping-pong state: subcycle k of a launch reads set (k & 1) and writes
  // set (k & 1) ^ 1 (a one-subcycle launch never writes set 0)
  double *u[2] = {}, *v[2] = {};
  double *s[2][12] = {};
  // written on the launch's last subcycle when `last` is set
  double *strintx = nullptr, *strinty = nullptr, *Cb = nullptr;
  double *str_out[8] = {};
  int nsub = 1;        // subcycles of this launch
  bool last = false;   // the launch's last subcycle is the call's last
  // Tape mode (uv_step > 0): subcycle k reads u[0] + k * uv_step and writes
  // u[0] + (k + 1) * uv_step (v likewise), so that every subcycle's
  // velocities stay in memory (the adjoint's tape entries); the stresses
  // still alternate between s[0] and s[1].
  size_t uv_step = 0;
  // A launch of several subcycles: per tile a counter that each consumer warp
  // raises by one when it is done with the tile in a subcycle (zeroed before
  // the launch), and the tiles each tile waits for (evp_tiles.h dep_off /
  // dep_idx) before it loads the next subcycle's state.
  unsigned *epoch = nullptr;
  const int32_t *dep_off = nullptr, *dep_idx = nullptr;
  int *err = nullptr;  // nonzero after a bounded wait ran out
  int prefetch = 0;    // tiles prefetched into L2 ahead of the shared ring
  // Launch as a programmatic dependent of the previous launch on the stream
  // (one-subcycle launches only).  The previous launch must be the preceding
  // subcycle's k_tma over the same plan: the dependent reads the records and
  // constant blocks before that launch has completed, the state after.
  bool pdl = false;
  // The stepu part may be the first kTmaStepuCompact fields (see there):
  // where `compact` is set, *cflags is 0 (the call's fields allow it; read
  // by the kernel, so captured launches stay valid across uploads) and
  // revp == 0 (checked at launch).
  bool compact = false;
  const int *cflags = nullptr;
  // optional timing trace of block 0 (debug): per tile 8 %globaltimer stamps
  // [0] producers issued all copies, [1] consumer 0 has the stress part,
  // [2] stress done (consumer barrier), [3] bulk warp has the tile record,
  // [4] stress slot free, [5] consumer warp 0 done with stepu, [6] bulk
  // copies issued, [7] gathers issued; kTraceTiles tiles at most
  long long *trace = nullptr;
};
constexpr int kTraceTiles = 256;

// Allow the kernel's dynamic shared memory (call once per device).
int tma_prepare(int device);
// binaryVersion of the subcycle kernel on the current device (100 = sm_100a).
cudaError_t tma_binary_version(int *version);
// What the wait that left `code` in the error word was waiting for.
const char *tma_wait_name(int code);
// One bounded wait on an mbarrier that nothing completes: it runs out after
// limit_ns and leaves its code in *err (a check of the timeout path).
void launch_wait_probe(int *err, unsigned long long limit_ns, cudaStream_t st);
// The same for the counter wait of a multi-subcycle launch: one wait on
// *counter (which must stay 0) that runs out after limit_ns.
void launch_dep_probe(int *err, const unsigned *counter, unsigned long long limit_ns,
                      cudaStream_t st);
// One CTA per run (grid = nruns, at most one per SM).  A launch of several
// subcycles (a.nsub > 1, a.epoch set) keeps its CTAs across the subcycles and
// needs them all resident at once: it is a cooperative launch.  Returns the
// launch's error.
cudaError_t launch_tma(const TmaArgs &a, const Params &p, cudaStream_t st);
// Whether this device runs several subcycles per launch (cooperative launch
// with one CTA per run resident on every SM).
bool tma_can_persist(int device, int nruns);

// ---- layout conversion between the reference 1D order and slots ----------
constexpr int kMaxBatch = 32;
struct PermBatch {
  int n = 0;
  const double *src[kMaxBatch] = {};
  double *dst[kMaxBatch] = {};
  double *dst2[kMaxBatch] = {};  // optional second copy (ping-pong buffers)
};
// dst[f][s] = src[f][point_of_slot[s]] (0 for padding slots), s < nslots.
void launch_scatter(const PermBatch &b, int nslots, const int32_t *point_of_slot,
                    cudaStream_t st);
// dst[f][p] = src[f][slot_of_point[p]], p < na.
void launch_gather(const PermBatch &b, int na, const int32_t *slot_of_point,
                   cudaStream_t st);
// flags[s] from int32 skipT/skipU in reference order (padding: both bits);
// meta[s] = lnb[s] | flags[s] << 30.
void launch_flags(int nslots, const int32_t *point_of_slot,
                  const int32_t *skipT, const int32_t *skipU, uint8_t *flags,
                  const uint32_t *lnb, uint32_t *meta, cudaStream_t st);
// cblk[(t*kConstFields + f)*256 + l] for l < tile_cnt[t] and slot
// s = tile_off[t] + l: src[f][s] for f < 7, meta[s] | lcor[s] << 32 with the
// sign bits of uinit (src[18]) and vinit (src[19]) in bits 62 and 63 for
// f = 7, src[f-1][s] for f >= 8; 0 for l >= tile_cnt[t].  *cflags gets bit 0
// if a Tbu (src[17]) is not +0 and bit 1 if a uinit or vinit is not finite.
void launch_const_blocks(int ntiles, const int32_t *tile_off, const int32_t *tile_cnt,
                         const double *const src[kConstFields - 1], const uint32_t *meta,
                         const uint32_t *lcor, double *cblk, int *cflags, cudaStream_t st);
// kvrel[s] = (aiu[s]*rhow)*Cw[s].
void launch_drag_factor(int nslots, const double *aiu, const double *Cw,
                        double rhow, double *kvrel, cudaStream_t st);

}  // namespace evp
