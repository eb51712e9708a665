// evp_kernels.cuh -- device data layout and kernel launchers of the EVP-1D
// library (internal, not part of the C-ABI).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "evp_math.cuh"

namespace evp {

// Skip flags packed per point: bit 0 = skipT, bit 1 = skipU.
constexpr uint8_t kSkipT = 1;
constexpr uint8_t kSkipU = 2;

// Device-resident problem in the reference's 1D order (0-based indices).
// uvel/vvel/str are navel long; the halo slots na..navel-1 of str stay 0.
struct DevState {
  int na = 0, navel = 0;
  const int32_t *ee = nullptr, *ne = nullptr, *se = nullptr;
  const int32_t *nw = nullptr, *sw = nullptr, *sse = nullptr;
  const uint8_t *flags = nullptr;
  // static geometry [na]
  const double *dxT = nullptr, *dyT = nullptr, *HTE = nullptr, *HTN = nullptr;
  const double *HTEm1 = nullptr, *HTNm1 = nullptr, *uarear = nullptr;
  // per-call inputs [na]
  const double *strength = nullptr, *Cw = nullptr, *aiu = nullptr;
  const double *uocn = nullptr, *vocn = nullptr, *waterx = nullptr;
  const double *watery = nullptr, *forcex = nullptr, *forcey = nullptr;
  const double *umassdti = nullptr, *fm = nullptr, *Tbu = nullptr;
  const double *uinit = nullptr, *vinit = nullptr;
  // state
  double *stress[12] = {};
  double *u = nullptr, *v = nullptr;  // [navel]
  double *str[8] = {};                // [navel]
  double *strintx = nullptr, *strinty = nullptr, *Cb = nullptr;
};

// One stress pass over all list points (src/bench_v2b.F90:62-312).
void launch_stress(const DevState &s, const Params &p, cudaStream_t st);
// One stepu pass over all list points (src/bench_v2b.F90:444-549).
void launch_stepu(const DevState &s, const Params &p, cudaStream_t st);

}  // namespace evp
