// evp1d_api.cu -- the C-ABI of include/evp1d.h: handle, validation, host<->
// device movement and the graph-launched subcycle loop.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "evp1d.h"
#include "evp_kernels.cuh"
#include "evp_internal.h"

using evp::DevState;
using evp::Params;

namespace {
thread_local std::string g_err;
}  // namespace

namespace evp {
int error(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}
}  // namespace evp

namespace {

#define fail evp::error

#define CUDA_TRY(x)                                                        \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess)                                                 \
      return fail(e_ == cudaErrorMemoryAllocation ? EVP1D_ERR_NOMEM        \
                                                  : EVP1D_ERR_CUDA,        \
                  "%s: %s", #x, cudaGetErrorString(e_));                   \
  } while (0)

#define CHECK(x) \
  do {           \
    int rc_ = (x); \
    if (rc_ != EVP1D_OK) return rc_; \
  } while (0)

Params to_params(const evp1d_params &q) {
  Params p;
  p.arlx1i = q.arlx1i;
  p.denom1 = q.denom1;
  p.brlx = q.brlx;
  p.capping = q.capping;
  p.e_factor = q.e_factor;
  p.epp2i = q.epp2i;
  p.deltaminEVP = q.deltaminEVP;
  p.revp = q.revp;
  p.Ktens = q.Ktens;
  p.u0 = q.u0;
  p.cosw = q.cosw;
  p.sinw = q.sinw;
  p.rhow = q.rhow;
  return p;
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// Number of subcycles captured in one CUDA graph.
constexpr int kGraphChunk = 50;

}  // namespace

struct evp1d_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  Params p{};
  DevState s{};
  void *arena = nullptr;
  size_t arena_bytes = 0;
  bool uploaded = false;
  bool have_str = false;  // str holds the result of a stress pass
  long long launches = 0;
  cudaGraphExec_t graph = nullptr;
  int graph_n = 0;
  std::vector<uint8_t> flags_host;
};

namespace {

int select_device(evp1d_t *h) {
  CUDA_TRY(cudaSetDevice(h->device));
  return EVP1D_OK;
}

void drop_graph(evp1d_t *h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
  h->graph_n = 0;
}

// Launch `n` subcycles of {stress; stepu} directly.
void launch_subcycles_direct(evp1d_t *h, int n) {
  for (int k = 0; k < n; k++) {
    evp::launch_stress(h->s, h->p, h->stream);
    evp::launch_stepu(h->s, h->p, h->stream);
  }
  h->launches += 2LL * n;
}

int build_graph(evp1d_t *h, int n) {
  drop_graph(h);
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < n; k++) {
    evp::launch_stress(h->s, h->p, h->stream);
    evp::launch_stepu(h->s, h->p, h->stream);
  }
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(EVP1D_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  }
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->graph = nullptr;
    return fail(EVP1D_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  }
  h->graph_n = n;
  return EVP1D_OK;
}

}  // namespace

extern "C" {

const char *evp1d_last_error(void) { return g_err.c_str(); }

const char *evp1d_version(void) { return "evp1d-b200 0.1 (sm_100a, fp64)"; }

void evp1d_set_evp_parameters(evp1d_params *p, int ndte) {
  // set_evp_parameters (src/ice.F90:109-130) with the fixed values of
  // src/ice.F90:80-90.
  const double e_plasticpot = 2.0, e_yieldcurve = 2.0, elasticDamp = 0.36;
  if (!p) return;
  p->u0 = 5e-5;
  p->cosw = 1.0;
  p->sinw = 0.0;
  p->Ktens = 0.0;
  p->revp = 0.0;
  p->rhow = 1026.0;
  p->epp2i = 1.0 / (e_plasticpot * e_plasticpot);
  p->capping = 1.0;
  p->e_factor = (e_yieldcurve * e_yieldcurve) /
                (e_plasticpot * e_plasticpot * e_plasticpot * e_plasticpot);
  const double arlx = 2.0 * elasticDamp * (double)ndte;
  p->arlx1i = 1.0 / arlx;
  p->brlx = (double)ndte;
  p->denom1 = 1.0 / (1.0 + p->arlx1i);
  p->deltaminEVP = 10e-9;
}

int evp1d_init(evp1d_t **handle, int na, int navel, const int32_t *ee,
               const int32_t *ne, const int32_t *se, const int32_t *nw,
               const int32_t *sw, const int32_t *sse, const double *dxT,
               const double *dyT, const double *HTE, const double *HTN,
               const double *HTEm1, const double *HTNm1, const double *uarear,
               const evp1d_params *params, int device) {
  g_err.clear();
  if (!handle) return fail(EVP1D_ERR_INVALID_ARG, "handle is NULL");
  *handle = nullptr;
  if (na < 0 || navel < na)
    return fail(EVP1D_ERR_INVALID_ARG, "need 0 <= na <= navel (na=%d navel=%d)",
                na, navel);
  if (!params) return fail(EVP1D_ERR_INVALID_ARG, "params is NULL");
  const int32_t *idx[6] = {ee, ne, se, nw, sw, sse};
  const double *geo[7] = {dxT, dyT, HTE, HTN, HTEm1, HTNm1, uarear};
  if (na > 0) {
    for (int k = 0; k < 6; k++)
      if (!idx[k]) return fail(EVP1D_ERR_INVALID_ARG, "neighbour vector %d is NULL", k);
    for (int k = 0; k < 7; k++)
      if (!geo[k]) return fail(EVP1D_ERR_INVALID_ARG, "geometry field %d is NULL", k);
  }
  // Host-side validation: every neighbour index must address a slot in
  // 1..navel, so no device gather can leave its buffer.
  static const char *nbname[6] = {"ee", "ne", "se", "nw", "sw", "sse"};
  for (int k = 0; k < 6; k++)
    for (int w = 0; w < na; w++) {
      const int32_t v = idx[k][w];
      if (v < 1 || v > navel)
        return fail(EVP1D_ERR_INDEX, "%s(%d) = %d outside 1..%d", nbname[k],
                    w + 1, (int)v, navel);
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return fail(EVP1D_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev)
    return fail(EVP1D_ERR_INVALID_ARG, "device %d not in 0..%d", device, ndev - 1);
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return fail(EVP1D_ERR_NO_DEVICE, "device %d is sm_%d%d; this build needs sm_100a",
                device, prop.major, prop.minor);

  evp1d_t *h = new evp1d_handle();
  h->device = device;
  h->p = to_params(*params);
  int rc = evp::internal_alloc(h->device, na, navel, &h->s, &h->arena,
                               &h->arena_bytes, &h->stream);
  if (rc != EVP1D_OK) {
    delete h;
    return rc;
  }
  rc = evp::internal_upload_static(h->s, idx, geo, h->stream);
  if (rc == EVP1D_OK) rc = select_device(h);
  if (rc == EVP1D_OK) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = fail(EVP1D_ERR_CUDA, "init: %s", cudaGetErrorString(e));
  }
  if (rc != EVP1D_OK) {
    evp1d_finalize(h);
    return rc;
  }
  *handle = h;
  return EVP1D_OK;
}

int evp1d_finalize(evp1d_t *h) {
  if (!h) return EVP1D_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  drop_graph(h);
  if (h->arena) cudaFree(h->arena);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return EVP1D_OK;
}

int evp1d_set_params(evp1d_t *h, const evp1d_params *params) {
  if (!h || !params) return fail(EVP1D_ERR_INVALID_ARG, "NULL argument");
  h->p = to_params(*params);
  drop_graph(h);
  return EVP1D_OK;
}

int evp1d_upload(evp1d_t *h, const evp1d_fields *io) {
  if (!h || !io) return fail(EVP1D_ERR_INVALID_ARG, "NULL argument");
  CHECK(select_device(h));
  CHECK(evp::internal_upload_fields(h->s, io, h->flags_host, h->stream));
  h->uploaded = true;
  h->have_str = false;
  return EVP1D_OK;
}

int evp1d_subcycles(evp1d_t *h, int ndte) {
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (ndte < 0) return fail(EVP1D_ERR_INVALID_ARG, "ndte = %d < 0", ndte);
  if (!h->uploaded) return fail(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  if (h->s.na == 0 || ndte == 0) return EVP1D_OK;
  CHECK(select_device(h));
  const int chunk = ndte < kGraphChunk ? ndte : kGraphChunk;
  const int full = ndte / chunk, rest = ndte - full * chunk;
  if (h->graph_n != chunk) CHECK(build_graph(h, chunk));
  for (int k = 0; k < full; k++) {
    CUDA_TRY(cudaGraphLaunch(h->graph, h->stream));
    h->launches += 2LL * chunk;
  }
  if (rest) launch_subcycles_direct(h, rest);
  CUDA_TRY(cudaGetLastError());
  h->have_str = true;
  return EVP1D_OK;
}

int evp1d_download(evp1d_t *h, const evp1d_fields *io) {
  if (!h || !io) return fail(EVP1D_ERR_INVALID_ARG, "NULL argument");
  if (!h->uploaded) return fail(EVP1D_ERR_STATE, "nothing uploaded");
  CHECK(select_device(h));
  return evp::internal_download_fields(h->s, io, h->stream);
}

int evp1d_run(evp1d_t *h, int ndte, const evp1d_fields *io) {
  CHECK(evp1d_upload(h, io));
  CHECK(evp1d_subcycles(h, ndte));
  return evp1d_download(h, io);
}

int evp1d_stress_only(evp1d_t *h, int n) {
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (n < 0) return fail(EVP1D_ERR_INVALID_ARG, "n = %d < 0", n);
  if (!h->uploaded) return fail(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  CHECK(select_device(h));
  for (int k = 0; k < n; k++) evp::launch_stress(h->s, h->p, h->stream);
  h->launches += h->s.na > 0 ? n : 0;
  CUDA_TRY(cudaGetLastError());
  if (n > 0) h->have_str = true;
  return EVP1D_OK;
}

int evp1d_stepu_only(evp1d_t *h, int n) {
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (n < 0) return fail(EVP1D_ERR_INVALID_ARG, "n = %d < 0", n);
  if (!h->uploaded) return fail(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  CHECK(select_device(h));
  for (int k = 0; k < n; k++) evp::launch_stepu(h->s, h->p, h->stream);
  h->launches += h->s.na > 0 ? n : 0;
  CUDA_TRY(cudaGetLastError());
  return EVP1D_OK;
}

int evp1d_synchronize(evp1d_t *h) {
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  CHECK(select_device(h));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return EVP1D_OK;
}

void *evp1d_stream(evp1d_t *h) { return h ? (void *)h->stream : nullptr; }

long long evp1d_launch_count(evp1d_t *h, int reset) {
  if (!h) return -1;
  long long n = h->launches;
  if (reset) h->launches = 0;
  return n;
}

}  // extern "C"
