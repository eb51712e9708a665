// evp_internal.h -- library-internal helpers shared by the C-ABI translation
// units (not part of the public ABI).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "evp1d.h"
#include "evp_kernels.cuh"

namespace evp {

// Record `fmt` as this thread's last error message and return `code`.
int error(int code, const char *fmt, ...);

// One device arena for the whole problem; fills the pointers of `s` and
// creates the handle's non-blocking stream.
int internal_alloc(int device, int na, int navel, DevState *s, void **arena,
                   size_t *bytes, cudaStream_t *stream);

// Neighbour vectors (1-based host -> 0-based device) and static geometry.
int internal_upload_static(const DevState &s, const int32_t *const idx[6],
                           const double *const geo[7], cudaStream_t st);

// Per-call fields host -> device; str is zeroed; uvel_init/vvel_init default
// to uvel/vvel.  `flags_host` is a reusable host buffer.
int internal_upload_fields(const DevState &s, const evp1d_fields *io,
                           std::vector<uint8_t> &flags_host, cudaStream_t st);

// Results device -> host; waits for the stream.
int internal_download_fields(const DevState &s, const evp1d_fields *io,
                             cudaStream_t st);

}  // namespace evp
