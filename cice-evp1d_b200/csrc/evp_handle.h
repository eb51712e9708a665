// evp_handle.h -- the evp1d_t handle shared by the C-ABI translation units
// (not part of the public ABI).
#pragma once

#include <string>
#include <vector>

#include "evp_internal.h"

struct evp1d_handle;
namespace evp {
struct AdjointState;
// Free the adjoint buffers of a handle (NULL is a no-op).
void adjoint_release(AdjointState *a);
// Free the velocity-exchange lists of a handle.
void exchange_release(evp1d_handle *h);
// Forget the recorded forward (the inputs or parameters changed).
void adjoint_invalidate(AdjointState *a);
}  // namespace evp

// Kernel paths of the fused subcycle.
enum { kPathTma = 0, kPathFused = 1 };

struct evp1d_handle {
  evp::DeviceProblem d;
  evp::Params p{};
  int path = kPathTma;
  int prefetch = 0;  // L2 prefetch distance of the TMA kernel (tiles)
  // TMA path: a call's subcycles in one launch whose CTAs stay resident
  // (cooperative), instead of one launch per subcycle in CUDA graphs
  bool persist = false;
  // TMA path: each subcycle's launch after the first of a call (and of a
  // captured chunk) is a programmatic dependent of the one before, so that
  // its prologue overlaps the previous launch's last tiles (EVP1D_PDL=0
  // turns it off)
  bool pdl = true;
  long long *trace = nullptr;  // device timing trace (EVP1D_TRACE, debug)
  bool uploaded = false;
  bool uinit_explicit = false;  // the last upload gave uvel_init/vvel_init
  long long launches = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // by starting buffer
  // ensemble (batched) handles: caller arrays are member-major concatenations
  // with each member's halo slots after its list points; uv_pos maps the
  // combined slot order (all list points, then all halo slots) to them.
  int nmembers = 1;
  std::vector<int64_t> uv_pos;
  std::vector<double> uv_tmp;  // scratch for u, v (and str) in combined order
  std::string tuned;           // last autotuner choice
  evp::AdjointState *adj = nullptr;  // checkpoints and work arrays of the adjoint
  // velocity exchange of a split state (evp1d_exchange_*): device positions
  // of the n_send sent points, then of the n_recv received ones
  int32_t *xpos = nullptr;
  double *xbuf = nullptr;  // in the same allocation: send, then receive buffer
  int nsend = 0, nrecv = 0;
};

