// evp_internal.h -- library-internal state shared by the C-ABI translation
// units (not part of the public ABI).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "evp1d.h"
#include "evp_kernels.cuh"
#include "evp_tiles.h"

namespace evp {

// Record `fmt` as this thread's last error message and return `code`.
int error(int code, const char *fmt, ...);

// A named NVTX range over a scope, so that the public calls show on a
// profiler's timeline (header-only NVTX; without a profiler it does nothing).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// Every device allocation of the library: cudaMalloc, unless the failure
// injection of evp1d_debug_fail_alloc picks this allocation, which then
// fails with cudaErrorMemoryAllocation and allocates nothing.
cudaError_t device_alloc(void **p, size_t bytes);
template <class T>
cudaError_t device_alloc(T **p, size_t bytes) {
  return device_alloc(reinterpret_cast<void **>(p), bytes);
}

// Per-call input fields in the order they are staged and scattered.
enum DynField {
  kStrength, kCw, kAiu, kUocn, kVocn, kWaterx, kWatery, kForcex, kForcey,
  kUmassdti, kFm, kTbu, kUinit, kVinit, kKvrel, kNumDyn
};
enum GeoField { kDxT, kDyT, kHTE, kHTN, kHTEm1, kHTNm1, kUarear, kNumGeo };

// The 1D problem on one GPU in slot order (tiles of the TilePlan), with the
// reference's halo slots appended after the nslots list slots for u, v, str.
struct DeviceProblem {
  int device = 0;
  cudaStream_t stream = nullptr;
  int na = 0, navel = 0, nslots = 0, nhs = 0, nuv = 0, ntiles = 0;
  bool from_coords = false;
  void *arena = nullptr;
  size_t arena_bytes = 0;
  // tile plan
  int nruns = 0;                 // CTAs of the subcycle kernel
  int32_t *run_off = nullptr;    // [nruns + 1] tile ranges of the runs
  int32_t *tile_off = nullptr, *tile_cnt = nullptr, *halo_off = nullptr;
  int32_t *halo_cnt = nullptr, *halo_idx = nullptr;
  int32_t *slot_of_point = nullptr, *point_of_slot = nullptr;
  int32_t *nb[6] = {};  // ee ne se nw sw sse, slot space
  uint32_t *lnb = nullptr;   // static packed stepu neighbours
  uint32_t *meta = nullptr;  // lnb | skip flags << 30 (per call)
  uint32_t *lcor = nullptr;  // packed stress corner velocity indices
  uint32_t *halo_lcc = nullptr, *halo_lcor = nullptr;
  int32_t *uvx_off = nullptr, *uvx_cnt = nullptr, *uvx_idx = nullptr;
  int32_t *dep_off = nullptr, *dep_idx = nullptr;  // subcycle dependencies (TilePlan)
  unsigned *epoch = nullptr;     // per-tile counters of a multi-subcycle launch
  int32_t *tile_meta = nullptr;  // 8 int32 per tile (see TmaArgs)
  int32_t *tile_rec = nullptr;   // kRecInts int32 per tile (producer records)
  double *cblk = nullptr;        // per-call constants, kConstFields x 256 per tile
  int *err = nullptr;        // device error word of the bounded waits
  // device word of launch_const_blocks' field checks: 0 when every Tbu of the
  // call is +0 and every uinit, vinit finite (TmaArgs::compact)
  int *cflags = nullptr;
  bool compact_allowed = true;  // EVP1D_COMPACT=0 at init turns the short part off
  int nctas = 0;             // SM count of the device
  uint8_t *flags = nullptr;
  double *geo[kNumGeo] = {};
  double *dyn[kNumDyn] = {};
  double *stress[2][12] = {};
  double *u[2] = {}, *v[2] = {};
  double *strintx = nullptr, *strinty = nullptr, *Cb = nullptr;
  double *str[8] = {};
  double *stage = nullptr;  // reference-order staging, 32 x navel doubles
  int cur = 0;              // buffer holding the current state
};

// Allocate and fill the static part from a tile plan and reference-order
// geometry (host).  Creates the stream.
int problem_create(DeviceProblem *d, int device, const TilePlan &plan,
                   const double *const geo[kNumGeo]);
void problem_destroy(DeviceProblem *d);

// Per-call fields host -> device (through the staging area); str zeroed;
// uvel_init/vvel_init default to the uploaded velocities; the drag factor
// (aiu*rhow)*Cw is precomputed; cur = 0.
int problem_upload(DeviceProblem *d, const evp1d_fields *io, double rhow);
// The device half of problem_upload: from the reference-order staging area
// (slots 0..11 per-call inputs, 12..23 stresses, 24 u, 25 v [navel], 26 uinit,
// 27 vinit, 28 strintx, 29 strinty, 30 Cb, 31 skipT then skipU as int32) into
// the slot-ordered state.
int problem_upload_staged(DeviceProblem *d, bool uinit_given, bool vinit_given, double rhow);
// The device half of problem_download: slot-ordered results into the staging
// area in reference order (slots 0..11 stresses, 12 u, 13 v, 14 strintx,
// 15 strinty, 16 Cb, 17 + k str_k when want_str[k]).
int problem_download_staged(DeviceProblem *d, const bool want_str[8]);
// Rebuild the per-tile constant blocks from the slot arrays (after the
// per-call fields or the drag factor changed), with the field checks in
// cflags.
int problem_fill_const(DeviceProblem *d);
// Results device -> host; waits for the stream.
int problem_download(DeviceProblem *d, const evp1d_fields *io);

// Views for the kernels.
DevState problem_inplace_view(const DeviceProblem &d);
FusedArgs problem_fused_args(const DeviceProblem &d, int from);
TmaArgs problem_tma_args(const DeviceProblem &d, int from);
// Read and clear the device error word (0 if no bounded wait ran out).
int problem_take_error(DeviceProblem *d, int *code);

}  // namespace evp
