// evp1d_api.cu -- the C-ABI of include/evp1d.h: handle, validation, host<->
// device movement and the graph-launched subcycle loop.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <atomic>
#include <cstring>
#include <string>
#include <vector>

#include "evp1d.h"
#include "evp_handle.h"
#include "evp_internal.h"

using evp::DevState;
using evp::DeviceProblem;
using evp::Params;

namespace {
thread_local std::string g_err;
// allocations left until the injected failure (0: none armed)
std::atomic<int> g_fail_alloc{0};
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

cudaError_t device_alloc(void **p, size_t bytes) {
  int n = g_fail_alloc.load();
  while (n > 0 && !g_fail_alloc.compare_exchange_weak(n, n - 1)) {
  }
  if (n == 1) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
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

#define CHECK(x)                    \
  do {                              \
    int rc_ = (x);                  \
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

// Subcycles per captured CUDA graph.  Even, so that a graph leaves the
// ping-pong parity unchanged.
constexpr int kGraphChunk = 50;

}  // namespace

namespace {

int select_device(evp1d_t *h) {
  CUDA_TRY(cudaSetDevice(h->d.device));
  return EVP1D_OK;
}

void drop_graphs(evp1d_t *h) {
  for (int k = 0; k < 2; k++) {
    if (h->graph[k]) cudaGraphExecDestroy(h->graph[k]);
    h->graph[k] = nullptr;
  }
}

// One subcycle from buffer `from` into the other one.  `after_sub`: the
// previous launch on the stream is this handle's previous subcycle (in the
// same call or the same captured chunk).
cudaError_t launch_sub(evp1d_t *h, int from, bool last, bool after_sub) {
  if (h->path == kPathTma) {
    evp::TmaArgs a = evp::problem_tma_args(h->d, from);
    a.prefetch = h->prefetch;
    a.trace = h->trace;
    a.nsub = 1;
    a.last = last;
    a.pdl = after_sub && h->pdl;
    return evp::launch_tma(a, h->p, h->d.stream);
  }
  evp::launch_fused(evp::problem_fused_args(h->d, from), h->p, last, h->d.stream);
  return cudaGetLastError();
}

// A bounded device-side wait that ran out leaves a code in the error word.
int check_device_error(evp1d_t *h) {
  int code = 0;
  CHECK(evp::problem_take_error(&h->d, &code));
  if (code)
    return fail(EVP1D_ERR_TIMEOUT,
                "a bounded device-side wait ran out (code %d: %s); the results of this "
                "call are not valid", code, evp::tma_wait_name(code));
  return EVP1D_OK;
}

// Capture kGraphChunk non-final fused subcycles starting from buffer `from`.
int build_graph(evp1d_t *h, int from) {
  cudaStream_t st = h->d.stream;
  cudaGraph_t g = nullptr;
  CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  int b = from;
  cudaError_t le = cudaSuccess;
  for (int k = 0; k < kGraphChunk && le == cudaSuccess; k++) {
    le = launch_sub(h, b, false, k > 0);
    b = 1 - b;
  }
  cudaError_t e = cudaStreamEndCapture(st, &g);
  if (e == cudaSuccess && le != cudaSuccess) e = le;
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(EVP1D_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  }
  e = cudaGraphInstantiate(&h->graph[from], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->graph[from] = nullptr;
    return fail(EVP1D_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  }
  return EVP1D_OK;
}

bool nonnull_all(const void *const *p, int n) {
  for (int k = 0; k < n; k++)
    if (!p[k]) return false;
  return true;
}

}  // namespace

extern "C" {

const char *evp1d_last_error(void) { return g_err.c_str(); }

int evp1d_host_alloc(void **ptr, size_t bytes) {
  if (!ptr) return fail(EVP1D_ERR_INVALID_ARG, "ptr is NULL");
  *ptr = nullptr;
  CUDA_TRY(cudaHostAlloc(ptr, bytes > 0 ? bytes : 1, cudaHostAllocPortable));
  return EVP1D_OK;
}

int evp1d_host_free(void *ptr) {
  if (ptr) CUDA_TRY(cudaFreeHost(ptr));
  return EVP1D_OK;
}

#ifndef EVP_TARGET
#define EVP_TARGET "unknown target"
#endif
const char *evp1d_version(void) {
  return "evp1d-b200 0.3 (" EVP_TARGET ", fp64, fused tile solver)";
}

int evp1d_binary_version(int device) {
  CUDA_TRY(cudaSetDevice(device));
  int v = 0;
  CUDA_TRY(evp::tma_binary_version(&v));
  return v;
}

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

}  // extern "C"

namespace {

int check_device(int device) {
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
    return fail(EVP1D_ERR_NO_DEVICE, "device %d is sm_%d%d; the library is compiled for sm_100a",
                device, prop.major, prop.minor);
  return EVP1D_OK;
}

// Largest tile compute set (points) of the plans of handles created from now
// on (evp1d_set_tile_points).
std::atomic<int> g_tile_points{evp::kTileCompute};

// Strip width of the grid order: EVP1D_STRIP_W (1..128), else 0 (the planner
// chooses by the points per run).
int strip_width() {
  if (const char *e = getenv("EVP1D_STRIP_W")) {
    const int v = atoi(e);
    if (v >= 1 && v <= 128) return v;
  }
  return 0;
}

// Runs (CTAs) of the plans made without a device: the B200's SM count.
constexpr int kDefaultRuns = 148;

// Validated 1-based neighbour vectors -> tile plan -> device problem.
int init_common(evp1d_t **handle, int na, int navel, const int32_t *const idx[6],
                const double *const geo[7], const evp1d_params *params, int device) {
  CHECK(check_device(device));
  std::vector<int32_t> nb0((size_t)na * 6);
  const int32_t *nbp[6];
  for (int k = 0; k < 6; k++) {
    for (int w = 0; w < na; w++) nb0[(size_t)k * na + w] = idx[k][w] - 1;
    nbp[k] = nb0.data() + (size_t)k * na;
  }
  int sms = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  // EVP1D_RUNS (1..SM count): fewer CTAs, for tests of the run boundaries
  if (const char *e = getenv("EVP1D_RUNS")) {
    const int v = atoi(e);
    if (v >= 1 && v < sms) sms = v;
  }
  evp::TilePlan plan;
  evp::build_tile_plan(na, navel, nbp, nullptr, nullptr, &plan, g_tile_points.load(), sms,
                       strip_width());
  if (getenv("EVP1D_CHECK_PLAN")) {
    std::string first;
    const long long bad = evp::verify_tile_plan(plan, nbp, g_tile_points.load(), &first);
    if (bad)
      return fail(EVP1D_ERR_INDEX, "tile plan: %lld violations, the first: %s", bad,
                  first.c_str());
  }

  evp1d_t *h = new evp1d_handle();
  h->p = to_params(*params);
  if (const char *e = getenv("EVP1D_PATH")) {
    if (!strcmp(e, "fused")) h->path = kPathFused;
  }
  if (getenv("EVP1D_TRACE")) {
    if (evp::device_alloc(&h->trace, sizeof(long long) * 8 * evp::kTraceTiles) != cudaSuccess)
      h->trace = nullptr;
    else
      cudaMemset(h->trace, 0, sizeof(long long) * 8 * evp::kTraceTiles);
  }
  if (const char *e = getenv("EVP1D_PREFETCH")) {
    const int v = atoi(e);
    h->prefetch = v < 0 ? 0 : (v > 8 ? 8 : v);
  }
  int rc = evp::problem_create(&h->d, device, plan, geo);
  if (rc != EVP1D_OK) {
    evp::problem_destroy(&h->d);
    if (h->trace) cudaFree(h->trace);
    delete h;
    return rc;
  }
  // EVP1D_PERSIST=1: a call's subcycles in one launch where the device keeps
  // every run's CTA resident (asked after problem_create has allowed the
  // kernel's shared memory).  Off by default: on grid1600x1200 it measured
  // 276 us per subcycle against 101 for one launch per subcycle, because a
  // run's first tile waits for the neighbouring runs' last tiles of the
  // subcycle before (the strip order chains the runs).
  if (const char *e = getenv("EVP1D_PERSIST"))
    h->persist = atoi(e) != 0 && evp::tma_can_persist(device, plan.nruns);
  if (const char *e = getenv("EVP1D_PDL")) h->pdl = atoi(e) != 0;
  if (const char *e = getenv("EVP1D_COMPACT")) h->d.compact_allowed = atoi(e) != 0;
  *handle = h;
  return EVP1D_OK;
}

int validate_neighbours(int na, int navel, const int32_t *const idx[6], int member) {
  static const char *nbname[6] = {"ee", "ne", "se", "nw", "sw", "sse"};
  for (int k = 0; k < 6; k++)
    for (int w = 0; w < na; w++) {
      const int32_t v = idx[k][w];
      if (v < 1 || v > navel) {
        if (member < 0)
          return fail(EVP1D_ERR_INDEX, "%s(%d) = %d outside 1..%d", nbname[k], w + 1, (int)v,
                      navel);
        return fail(EVP1D_ERR_INDEX, "member %d: %s(%d) = %d outside 1..%d", member,
                    nbname[k], w + 1, (int)v, navel);
      }
    }
  return EVP1D_OK;
}

// Fields of a batched handle with u, v (and str) reordered into the combined
// slot order; `io` is the caller's member-major layout.
evp1d_fields combined_view(evp1d_t *h, const evp1d_fields *io, bool fill) {
  evp1d_fields c = *io;
  const size_t nv = h->uv_pos.size();
  int nstr = 0;
  for (int k = 0; k < 8; k++) nstr += io->str[k] ? 1 : 0;
  h->uv_tmp.resize(nv * (size_t)(2 + nstr));
  double *u = h->uv_tmp.data(), *v = u + nv;
  if (fill) {
    for (size_t k = 0; k < nv; k++) {
      u[k] = io->uvel[h->uv_pos[k]];
      v[k] = io->vvel[h->uv_pos[k]];
    }
  }
  c.uvel = u;
  c.vvel = v;
  int q = 0;
  for (int k = 0; k < 8; k++) c.str[k] = io->str[k] ? u + (size_t)(2 + q++) * nv : nullptr;
  return c;
}

void scatter_combined(evp1d_t *h, const evp1d_fields *io, int na_total) {
  const size_t nv = h->uv_pos.size();
  const double *u = h->uv_tmp.data(), *v = u + nv;
  for (int k = 0; k < na_total; k++) {  // list slots are updated; halo slots are not
    io->uvel[h->uv_pos[k]] = u[k];
    io->vvel[h->uv_pos[k]] = v[k];
  }
  int q = 0;
  for (int k = 0; k < 8; k++)
    if (io->str[k]) {
      const double *s = u + (size_t)(2 + q++) * nv;
      for (size_t w = 0; w < nv; w++) io->str[k][h->uv_pos[w]] = s[w];
    }
}

}  // namespace

extern "C" {

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
    if (!nonnull_all((const void *const *)idx, 6))
      return fail(EVP1D_ERR_INVALID_ARG, "a neighbour vector is NULL");
    if (!nonnull_all((const void *const *)geo, 7))
      return fail(EVP1D_ERR_INVALID_ARG, "a geometry field is NULL");
  }
  // Host-side validation: every neighbour index must address a slot in
  // 1..navel, so no device gather can leave its buffer.
  CHECK(validate_neighbours(na, navel, idx, -1));
  return init_common(handle, na, navel, idx, geo, params, device);
}

int evp1d_init_batched(evp1d_t **handle, int nmembers, const int32_t *na_m,
                       const int32_t *navel_m, const int32_t *ee, const int32_t *ne,
                       const int32_t *se, const int32_t *nw, const int32_t *sw,
                       const int32_t *sse, const double *dxT, const double *dyT,
                       const double *HTE, const double *HTN, const double *HTEm1,
                       const double *HTNm1, const double *uarear,
                       const evp1d_params *params, int device) {
  g_err.clear();
  if (!handle) return fail(EVP1D_ERR_INVALID_ARG, "handle is NULL");
  *handle = nullptr;
  if (nmembers < 1 || !na_m || !navel_m || !params)
    return fail(EVP1D_ERR_INVALID_ARG, "need nmembers >= 1, na, navel and params");
  long long NA = 0, NV = 0;
  for (int m = 0; m < nmembers; m++) {
    if (na_m[m] < 0 || navel_m[m] < na_m[m])
      return fail(EVP1D_ERR_INVALID_ARG, "member %d: need 0 <= na <= navel", m);
    NA += na_m[m];
    NV += navel_m[m];
  }
  if (NV > 0x7fffffffLL) return fail(EVP1D_ERR_INVALID_ARG, "ensemble too large for int32");
  const int32_t *idx[6] = {ee, ne, se, nw, sw, sse};
  const double *geo[7] = {dxT, dyT, HTE, HTN, HTEm1, HTNm1, uarear};
  if (NA > 0) {
    if (!nonnull_all((const void *const *)idx, 6))
      return fail(EVP1D_ERR_INVALID_ARG, "a neighbour vector is NULL");
    if (!nonnull_all((const void *const *)geo, 7))
      return fail(EVP1D_ERR_INVALID_ARG, "a geometry field is NULL");
  }
  // combined 1-based index space: all members' list points, then all halos
  std::vector<int32_t> comb((size_t)NA * 6);
  std::vector<int64_t> uv_pos((size_t)NV);
  long long lo = 0, ho = 0, co = 0;  // list offset, halo offset, caller offset
  for (int m = 0; m < nmembers; m++) {
    const int n = na_m[m], nv = navel_m[m];
    const int32_t *mi[6];
    for (int k = 0; k < 6; k++) mi[k] = idx[k] + lo;
    CHECK(validate_neighbours(n, nv, mi, m));
    for (int k = 0; k < 6; k++)
      for (int w = 0; w < n; w++) {
        const int32_t v = mi[k][w];
        comb[(size_t)k * NA + lo + w] = (int32_t)(v <= n ? lo + v : NA + ho + (v - n));
      }
    for (int w = 0; w < n; w++) uv_pos[lo + w] = co + w;
    for (int w = 0; w < nv - n; w++) uv_pos[NA + ho + w] = co + n + w;
    lo += n;
    ho += nv - n;
    co += nv;
  }
  const int32_t *cidx[6];
  for (int k = 0; k < 6; k++) cidx[k] = comb.data() + (size_t)k * NA;
  CHECK(init_common(handle, (int)NA, (int)NV, cidx, geo, params, device));
  (*handle)->nmembers = nmembers;
  (*handle)->uv_pos = std::move(uv_pos);
  return EVP1D_OK;
}

int evp1d_finalize(evp1d_t *h) {
  if (!h) return EVP1D_OK;
  cudaSetDevice(h->d.device);
  drop_graphs(h);
  evp::adjoint_release(h->adj);
  evp::exchange_release(h);
  evp::problem_destroy(&h->d);
  if (h->trace) cudaFree(h->trace);
  delete h;
  return EVP1D_OK;
}

int evp1d_set_params(evp1d_t *h, const evp1d_params *params) {
  if (!h || !params) return fail(EVP1D_ERR_INVALID_ARG, "NULL argument");
  CHECK(select_device(h));
  const double old_rhow = h->p.rhow;
  h->p = to_params(*params);
  drop_graphs(h);
  evp::adjoint_invalidate(h->adj);
  if (h->uploaded && h->p.rhow != old_rhow && h->d.nslots > 0) {
    evp::launch_drag_factor(h->d.nslots, h->d.dyn[evp::kAiu], h->d.dyn[evp::kCw],
                            h->p.rhow, h->d.dyn[evp::kKvrel], h->d.stream);
    CHECK(evp::problem_fill_const(&h->d));
  }
  return EVP1D_OK;
}

int evp1d_upload(evp1d_t *h, const evp1d_fields *io) {
  evp::NvtxRange nvtx_range("evp1d_upload");
  if (!h || !io) return fail(EVP1D_ERR_INVALID_ARG, "NULL argument");
  CHECK(select_device(h));
  evp::adjoint_invalidate(h->adj);
  h->uinit_explicit = io->uvel_init != nullptr;
  if (h->nmembers > 1 && h->d.na > 0) {
    if (!io->uvel || !io->vvel) return fail(EVP1D_ERR_INVALID_ARG, "uvel/vvel are NULL");
    const evp1d_fields c = combined_view(h, io, true);
    CHECK(evp::problem_upload(&h->d, &c, h->p.rhow));
  } else {
    CHECK(evp::problem_upload(&h->d, io, h->p.rhow));
  }
  h->uploaded = true;
  return EVP1D_OK;
}

}  // extern "C"

namespace {
// ndte subcycles; `ends` = the last one ends the call (writes strintx,
// strinty, Cb and str).
int run_subcycles(evp1d_t *h, int ndte, bool ends) {
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (ndte < 0) return fail(EVP1D_ERR_INVALID_ARG, "ndte = %d < 0", ndte);
  if (!h->uploaded) return fail(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  if (h->d.ntiles == 0 || ndte == 0) return EVP1D_OK;
  CHECK(select_device(h));
  cudaStream_t st = h->d.stream;
  if (h->path == kPathTma && h->persist && ndte > 1) {
    // the whole call in one launch; the per-tile counters start at zero
    CUDA_TRY(cudaMemsetAsync(h->d.epoch, 0, sizeof(unsigned) * (size_t)h->d.ntiles, st));
    evp::TmaArgs a = evp::problem_tma_args(h->d, h->d.cur);
    a.trace = h->trace;
    a.nsub = ndte;
    a.last = ends;
    a.epoch = h->d.epoch;
    CUDA_TRY(evp::launch_tma(a, h->p, st));
    if (ndte & 1) h->d.cur = 1 - h->d.cur;
    h->launches++;
    return EVP1D_OK;
  }
  int body = ndte - 1;  // subcycles before the last one
  while (body >= kGraphChunk) {
    const int c = h->d.cur;
    if (!h->graph[c]) CHECK(build_graph(h, c));
    CUDA_TRY(cudaGraphLaunch(h->graph[c], st));
    h->launches += kGraphChunk;
    body -= kGraphChunk;
  }
  // a launch right after a graph launch waits for the whole graph
  bool after_sub = false;
  for (; body > 0; body--) {
    CUDA_TRY(launch_sub(h, h->d.cur, false, after_sub));
    after_sub = true;
    h->d.cur = 1 - h->d.cur;
    h->launches++;
  }
  CUDA_TRY(launch_sub(h, h->d.cur, ends, after_sub));
  h->d.cur = 1 - h->d.cur;
  h->launches++;
  CUDA_TRY(cudaGetLastError());
  return EVP1D_OK;
}
}  // namespace

extern "C" {

int evp1d_subcycles(evp1d_t *h, int ndte) {
  evp::NvtxRange nvtx_range("evp1d_subcycles");
  return run_subcycles(h, ndte, true);
}

int evp1d_subcycles_inner(evp1d_t *h, int n) {
  evp::NvtxRange nvtx_range("evp1d_subcycles_inner");
  return run_subcycles(h, n, false);
}

int evp1d_download(evp1d_t *h, const evp1d_fields *io) {
  evp::NvtxRange nvtx_range("evp1d_download");
  if (!h || !io) return fail(EVP1D_ERR_INVALID_ARG, "NULL argument");
  if (!h->uploaded) return fail(EVP1D_ERR_STATE, "nothing uploaded");
  CHECK(select_device(h));
  CHECK(check_device_error(h));
  if (h->nmembers > 1 && h->d.na > 0) {
    if (!io->uvel || !io->vvel) return fail(EVP1D_ERR_INVALID_ARG, "uvel/vvel are NULL");
    const evp1d_fields c = combined_view(h, io, false);
    CHECK(evp::problem_download(&h->d, &c));
    scatter_combined(h, io, h->d.na);
    return EVP1D_OK;
  }
  return evp::problem_download(&h->d, io);
}

int evp1d_run(evp1d_t *h, int ndte, const evp1d_fields *io) {
  evp::NvtxRange nvtx_range("evp1d_run");
  CHECK(evp1d_upload(h, io));
  CHECK(evp1d_subcycles(h, ndte));
  return evp1d_download(h, io);
}

int evp1d_stress_only(evp1d_t *h, int n) {
  evp::NvtxRange nvtx_range("evp1d_stress_only");
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (n < 0) return fail(EVP1D_ERR_INVALID_ARG, "n = %d < 0", n);
  if (!h->uploaded) return fail(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  if (h->d.nslots == 0) return EVP1D_OK;
  CHECK(select_device(h));
  const DevState s = evp::problem_inplace_view(h->d);
  for (int k = 0; k < n; k++) evp::launch_stress(s, h->p, h->d.stream);
  h->launches += n;
  CUDA_TRY(cudaGetLastError());
  return EVP1D_OK;
}

int evp1d_stepu_only(evp1d_t *h, int n) {
  evp::NvtxRange nvtx_range("evp1d_stepu_only");
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (n < 0) return fail(EVP1D_ERR_INVALID_ARG, "n = %d < 0", n);
  if (!h->uploaded) return fail(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  if (h->d.nslots == 0) return EVP1D_OK;
  CHECK(select_device(h));
  const DevState s = evp::problem_inplace_view(h->d);
  for (int k = 0; k < n; k++) evp::launch_stepu(s, h->p, h->d.stream);
  h->launches += n;
  CUDA_TRY(cudaGetLastError());
  return EVP1D_OK;
}

int evp1d_synchronize(evp1d_t *h) {
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  CHECK(select_device(h));
  CUDA_TRY(cudaStreamSynchronize(h->d.stream));
  return check_device_error(h);
}

int evp1d_set_tile_points(int points) {
  if (points < 32 || points > evp::kTileCompute)
    return fail(EVP1D_ERR_INVALID_ARG, "tile points %d outside [32, %d]", points,
                evp::kTileCompute);
  g_tile_points.store(points);
  return EVP1D_OK;
}

int evp1d_get_tile_points(void) { return g_tile_points.load(); }

int evp1d_debug_wait_timeout(evp1d_t *h, long long ns) {
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (ns < 1000000 || ns > 1000000000)
    return fail(EVP1D_ERR_INVALID_ARG, "wait limit %lld ns outside [1e6, 1e9]", ns);
  CUDA_TRY(cudaSetDevice(h->d.device));
  evp::launch_wait_probe(h->d.err, (unsigned long long)ns, h->d.stream);
  CUDA_TRY(cudaGetLastError());
  return EVP1D_OK;
}

int evp1d_debug_dep_wait_timeout(evp1d_t *h, long long ns) {
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (ns < 1000000 || ns > 1000000000)
    return fail(EVP1D_ERR_INVALID_ARG, "wait limit %lld ns outside [1e6, 1e9]", ns);
  if (h->d.ntiles == 0) return fail(EVP1D_ERR_STATE, "the problem has no tiles");
  CUDA_TRY(cudaSetDevice(h->d.device));
  // the first tile's counter, zeroed here and raised by no kernel meanwhile
  CUDA_TRY(cudaMemsetAsync(h->d.epoch, 0, sizeof(unsigned), h->d.stream));
  evp::launch_dep_probe(h->d.err, h->d.epoch, (unsigned long long)ns, h->d.stream);
  CUDA_TRY(cudaGetLastError());
  return EVP1D_OK;
}

int evp1d_debug_fail_alloc(int n) {
  if (n < 0) return fail(EVP1D_ERR_INVALID_ARG, "n = %d < 0", n);
  g_fail_alloc.store(n);
  return EVP1D_OK;
}

int evp1d_debug_trace(evp1d_t *h, long long *out, int n) {
  if (!h || !out || n < 0) return fail(EVP1D_ERR_INVALID_ARG, "bad arguments");
  if (!h->trace) return fail(EVP1D_ERR_STATE, "tracing is off (set EVP1D_TRACE)");
  if (n > 8 * evp::kTraceTiles) n = 8 * evp::kTraceTiles;
  CHECK(select_device(h));
  CUDA_TRY(cudaStreamSynchronize(h->d.stream));
  CUDA_TRY(cudaMemcpy(out, h->trace, sizeof(long long) * (size_t)n, cudaMemcpyDeviceToHost));
  return EVP1D_OK;
}

int evp1d_autotune(evp1d_t *h, int nsub, char *chosen, int len) {
  if (!h) return fail(EVP1D_ERR_INVALID_ARG, "NULL handle");
  if (nsub < 1) return fail(EVP1D_ERR_INVALID_ARG, "nsub = %d < 1", nsub);
  if (!h->uploaded) return fail(EVP1D_ERR_STATE, "evp1d_upload has not been called");
  CHECK(select_device(h));
  DeviceProblem &d = h->d;
  if (d.ntiles == 0) return EVP1D_OK;
  cudaStream_t st = d.stream;
  // every array a trial writes: both state buffers, outputs, str
  std::vector<std::pair<double *, size_t>> arrs;
  for (int b = 0; b < 2; b++) {
    for (int k = 0; k < 12; k++) arrs.push_back({d.stress[b][k], (size_t)d.nslots});
    arrs.push_back({d.u[b], (size_t)d.nuv});
    arrs.push_back({d.v[b], (size_t)d.nuv});
  }
  arrs.push_back({d.strintx, (size_t)d.nslots});
  arrs.push_back({d.strinty, (size_t)d.nslots});
  arrs.push_back({d.Cb, (size_t)d.nslots});
  for (int k = 0; k < 8; k++) arrs.push_back({d.str[k], (size_t)d.nuv});
  size_t total = 0;
  for (auto &a : arrs) total += a.second;
  double *backup = nullptr;
  CUDA_TRY(evp::device_alloc(&backup, total * sizeof(double)));
  auto copy_all = [&](bool save) {
    size_t o = 0;
    for (auto &a : arrs) {
      if (save)
        cudaMemcpyAsync(backup + o, a.first, a.second * sizeof(double), cudaMemcpyDeviceToDevice, st);
      else
        cudaMemcpyAsync(a.first, backup + o, a.second * sizeof(double), cudaMemcpyDeviceToDevice, st);
      o += a.second;
    }
  };
  const int cur0 = d.cur;
  copy_all(true);
  struct Cand {
    int path, prefetch;
    bool persist;
  };
  // the multi-subcycle launch (EVP1D_PERSIST) stays a caller's choice: it is
  // far slower with the strip-ordered runs
  const Cand all[] = {{kPathTma, 0, false}, {kPathTma, 2, false}, {kPathFused, 0, false}};
  std::vector<Cand> cands(all, all + 3);
  const int old_path = h->path, old_pf = h->prefetch;
  const bool old_persist = h->persist;
  int best = -1;
  float best_ms = 0.f;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = EVP1D_OK;
  for (int c = 0; c < (int)cands.size() && rc == EVP1D_OK; c++) {
    h->path = cands[c].path;
    h->prefetch = cands[c].prefetch;
    h->persist = cands[c].persist;
    drop_graphs(h);
    rc = evp1d_subcycles(h, 2);  // warm-up (also builds nothing: < one chunk)
    if (rc == EVP1D_OK) {
      cudaEventRecord(e0, st);
      rc = evp1d_subcycles(h, nsub);
      cudaEventRecord(e1, st);
    }
    if (rc != EVP1D_OK) {
      // put the caller's state back before reporting the failed trial
      copy_all(false);
      d.cur = cur0;
      break;
    }
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (best < 0 || ms < best_ms) {
      best = c;
      best_ms = ms;
    }
    copy_all(false);
    d.cur = cur0;
  }
  cudaStreamSynchronize(st);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(backup);
  drop_graphs(h);
  if (rc != EVP1D_OK || best < 0) {
    h->path = old_path;
    h->prefetch = old_pf;
    h->persist = old_persist;
    return rc != EVP1D_OK ? rc : fail(EVP1D_ERR_CUDA, "autotune found no candidate");
  }
  CHECK(check_device_error(h));
  h->path = cands[best].path;
  h->prefetch = cands[best].prefetch;
  h->persist = cands[best].persist;
  char buf[128];
  snprintf(buf, sizeof buf, "%s%s prefetch=%d (%.2f us/subcycle)",
           h->path == kPathTma ? "fused-tile-tma" : "fused-tile",
           h->persist ? " multi-subcycle" : "", h->prefetch, 1000.0 * best_ms / nsub);
  h->tuned = buf;
  if (chosen && len > 0) {
    strncpy(chosen, buf, (size_t)len - 1);
    chosen[len - 1] = 0;
  }
  return EVP1D_OK;
}

const char *evp1d_kernel_path(evp1d_t *h) {
  if (!h) return "";
  return h->path == kPathTma ? "fused-tile-tma" : "fused-tile";
}

namespace {
// The host half of evp1d_init for the plan diagnostics: checked 1-based
// neighbour vectors -> 0-based copies (nb0, nbp) -> the tile plan.
int plan_from_vectors(int na, int navel, const int32_t *const idx[6], std::vector<int32_t> &nb0,
                      const int32_t *nbp[6], evp::TilePlan *plan) {
  if (na < 0 || navel < na) return fail(EVP1D_ERR_INVALID_ARG, "bad arguments");
  if (na > 0 && !nonnull_all((const void *const *)idx, 6))
    return fail(EVP1D_ERR_INVALID_ARG, "a neighbour vector is NULL");
  nb0.assign((size_t)na * 6, 0);
  for (int k = 0; k < 6; k++) {
    for (int w = 0; w < na; w++) {
      const int32_t v = idx[k][w];
      if (v < 1 || v > navel) return fail(EVP1D_ERR_INDEX, "index out of range");
      nb0[(size_t)k * na + w] = v - 1;
    }
    nbp[k] = nb0.data() + (size_t)k * na;
  }
  evp::build_tile_plan(na, navel, nbp, nullptr, nullptr, plan, g_tile_points.load(),
                       kDefaultRuns, strip_width());
  return EVP1D_OK;
}
}  // namespace

int evp1d_plan_check(int na, int navel, const int32_t *ee, const int32_t *ne,
                     const int32_t *se, const int32_t *nw, const int32_t *sw,
                     const int32_t *sse, long long *violations) {
  const int32_t *idx[6] = {ee, ne, se, nw, sw, sse};
  std::vector<int32_t> nb0;
  const int32_t *nbp[6] = {};
  evp::TilePlan plan;
  CHECK(plan_from_vectors(na, navel, idx, nb0, nbp, &plan));
  std::string first;
  const long long bad = evp::verify_tile_plan(plan, nbp, g_tile_points.load(), &first);
  if (violations) *violations = bad;
  if (bad)
    return fail(EVP1D_ERR_INDEX, "tile plan: %lld violations, the first: %s", bad, first.c_str());
  return EVP1D_OK;
}

int evp1d_plan_stats(int na, int navel, const int32_t *ee, const int32_t *ne,
                     const int32_t *se, const int32_t *nw, const int32_t *sw,
                     const int32_t *sse, long long stats[8]) {
  if (!stats) return fail(EVP1D_ERR_INVALID_ARG, "bad arguments");
  const int32_t *idx[6] = {ee, ne, se, nw, sw, sse};
  std::vector<int32_t> nb0;
  const int32_t *nbp[6] = {};
  evp::TilePlan plan;
  CHECK(plan_from_vectors(na, navel, idx, nb0, nbp, &plan));
  long long hmax = 0, tmax = 0, xmax = 0, rmax = 0;
  for (int t = 0; t < plan.ntiles; t++) {
    if (plan.halo_cnt[t] > hmax) hmax = plan.halo_cnt[t];
    if (plan.tile_cnt[t] > tmax) tmax = plan.tile_cnt[t];
    if (plan.uvx_cnt[t] > xmax) xmax = plan.uvx_cnt[t];
  }
  for (int r = 0; r < plan.nruns; r++)
    rmax = std::max<long long>(rmax, plan.run_off[r + 1] - plan.run_off[r]);
  for (int k = 0; k < 8; k++) stats[k] = 0;
  stats[0] = plan.ntiles;
  stats[1] = plan.nslots;
  stats[2] = (long long)plan.halo_idx.size();
  stats[3] = plan.from_coords ? 1 : 0;
  stats[4] = hmax;
  stats[5] = tmax;
  stats[6] = xmax;
  stats[7] = rmax;
  return EVP1D_OK;
}

void *evp1d_stream(evp1d_t *h) { return h ? (void *)h->d.stream : nullptr; }

long long evp1d_launch_count(evp1d_t *h, int reset) {
  if (!h) return -1;
  long long n = h->launches;
  if (reset) h->launches = 0;
  return n;
}

}  // extern "C"
