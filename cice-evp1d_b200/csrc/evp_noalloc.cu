// evp_noalloc.cu -- evp1d_run_device_noalloc: the subcycle loop on caller-owned
// device arrays in the reference 1D layout, for callers that cannot allocate
// device memory (a host code whose device memory is owned by another runtime
// or memory pool, or that runs where a cudaMalloc would synchronise or fail).
//
// It runs the reference-order pair of grid-stride kernels (stress then stepu,
// src/bench_v2b.F90:62-312, 444-549; the loop of
// integration/ice_dyn_evp1d.F90:188-207) in place on the caller's arrays.
// The only scratch -- str1..str8 and the velocities at call start -- lives in
// one file-scope device array of fixed size, so the call allocates nothing.
#include <cstdint>

#include "evp1d.h"
#include "evp_internal.h"

namespace evp {
namespace {

constexpr int kThreads = 256;

// Largest navel the scratch holds, and its layout: str1..str8, uvel at call
// start, vvel at call start, each kNoAllocMaxNavel doubles (20 MiB in all).
constexpr int kNoAllocMaxNavel = EVP1D_NOALLOC_MAX_NAVEL;
constexpr int kScratchArrays = 10;
// The check's "no bad neighbour" value: every byte 0x7f (one cudaMemsetAsync),
// above any 1 + point index since navel <= kNoAllocMaxNavel.
constexpr int kStatusNone = 0x7f7f7f7f;

static __device__ __align__(256) double g_scratch[kScratchArrays * (size_t)kNoAllocMaxNavel];
// Index-check result of the current call (0 = every neighbour in range).
static __device__ __align__(256) int g_status[1];

struct NaArgs {
  int na, navel;
  const int32_t *ee, *ne, *se, *nw, *sw, *sse;  // 1-based, as the reference
  const int32_t *skipT, *skipU;                 // nonzero = skip
  const double *dxT, *dyT, *HTE, *HTN, *HTEm1, *HTNm1, *uarear;
  const double *strength, *Cw, *aiu, *uocn, *vocn, *waterx, *watery;
  const double *forcex, *forcey, *umassdti, *fm, *Tbu;
  const double *uinit, *vinit;
  double *stress[12];
  double *u, *v;
  double *str[8];  // the scratch
  double *strintx, *strinty, *Cb;
};

// Flags any neighbour outside 1..navel: status[0], which starts at
// kStatusNone, ends as 1 + the lowest 0-based point with a bad neighbour.
__global__ void __launch_bounds__(kThreads) k_na_check(NaArgs a, int *status) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < a.na;
       w += gridDim.x * blockDim.x) {
    const int32_t *nb[6] = {a.ee, a.ne, a.se, a.nw, a.sw, a.sse};
    bool bad = false;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const int32_t x = nb[k][w];
      bad |= x < 1 || x > a.navel;
    }
    if (bad) atomicMin(status, w + 1);
  }
}

// At most 128 registers: two blocks (16 warps) per SM.
__global__ void __launch_bounds__(kThreads, 2) k_na_stress(NaArgs a, Params p) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < a.na;
       w += gridDim.x * blockDim.x) {
    if (a.skipT[w]) continue;
    const int iee = a.ee[w] - 1, ine = a.ne[w] - 1, ise = a.se[w] - 1;
    Corners c;
    c.ucc = a.u[w];
    c.vcc = a.v[w];
    c.uee = a.u[iee];
    c.vee = a.v[iee];
    c.une = a.u[ine];
    c.vne = a.v[ine];
    c.use = a.u[ise];
    c.vse = a.v[ise];
    const Geom g = make_geom(a.dxT[w], a.dyT[w], a.HTE[w], a.HTN[w], a.HTEm1[w],
                             a.HTNm1[w], p.deltaminEVP);
    const Strain sr = strain_rates(c, g, p.e_factor);
    double st[12], out[8];
#pragma unroll
    for (int k = 0; k < 12; k++) st[k] = a.stress[k][w];
    stress_update(st, out, sr, a.strength[w], g, p);
#pragma unroll
    for (int k = 0; k < 12; k++) a.stress[k][w] = st[k];
#pragma unroll
    for (int k = 0; k < 8; k++) a.str[k][w] = out[k];
  }
}

__global__ void __launch_bounds__(kThreads) k_na_stepu(NaArgs a, Params p) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < a.na;
       w += gridDim.x * blockDim.x) {
    if (a.skipU[w]) continue;
    const int inw = a.nw[w] - 1, isw = a.sw[w] - 1, isse = a.sse[w] - 1;
    StepuIn in;
    in.uold = a.u[w];
    in.vold = a.v[w];
    in.kvrel = drag_factor(a.aiu[w], p.rhow, a.Cw[w]);
    in.uocn = a.uocn[w];
    in.vocn = a.vocn[w];
    in.waterx = a.waterx[w];
    in.watery = a.watery[w];
    in.forcex = a.forcex[w];
    in.forcey = a.forcey[w];
    in.umassdti = a.umassdti[w];
    in.fm = a.fm[w];
    in.uarear = a.uarear[w];
    in.Tbu = a.Tbu[w];
    in.uinit = a.uinit[w];
    in.vinit = a.vinit[w];
    in.s1 = a.str[0][w];
    in.s2nw = a.str[1][inw];
    in.s3sse = a.str[2][isse];
    in.s4sw = a.str[3][isw];
    in.s5 = a.str[4][w];
    in.s6sse = a.str[5][isse];
    in.s7nw = a.str[6][inw];
    in.s8sw = a.str[7][isw];
    const StepuOut o = stepu_point(in, p);
    a.Cb[w] = o.Cb;
    a.strintx[w] = o.strintx;
    a.strinty[w] = o.strinty;
    a.u[w] = o.u;
    a.v[w] = o.v;
  }
}

#define NA_TRY(x)                                                          \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess)                                                 \
      return error(EVP1D_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_));  \
  } while (0)

// Device addresses of the scratch in the current context.  Looked up on
// every call: the module holding the arrays is loaded once per context, so
// after a cudaDeviceReset, or in a context other than the primary one, the
// arrays can sit at another address than in an earlier call.  The lookup
// allocates nothing once the module is loaded.
int scratch_in_context(double **scratch, int **status) {
  void *ps = nullptr, *pe = nullptr;
  NA_TRY(cudaGetSymbolAddress(&ps, g_scratch));
  NA_TRY(cudaGetSymbolAddress(&pe, g_status));
  *scratch = static_cast<double *>(ps);
  *status = static_cast<int *>(pe);
  return EVP1D_OK;
}

// A device pointer of the current device (or managed memory).
int check_device_ptr(const void *ptr, int dev, const char *name) {
  if (!ptr) return error(EVP1D_ERR_INVALID_ARG, "%s is NULL", name);
  cudaPointerAttributes at;
  const cudaError_t e = cudaPointerGetAttributes(&at, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return error(EVP1D_ERR_INVALID_ARG, "%s: not a CUDA pointer (%s)", name,
                 cudaGetErrorString(e));
  }
  if (at.type == cudaMemoryTypeManaged) return EVP1D_OK;
  if (at.type != cudaMemoryTypeDevice || at.device != dev)
    return error(EVP1D_ERR_INVALID_ARG,
                 "%s is not device memory of the current device %d", name, dev);
  return EVP1D_OK;
}

Params kernel_params(const evp1d_params &q) {
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

int grid_for(int n) {
  const int b = (n + kThreads - 1) / kThreads;
  return b < 1 ? 1 : b;
}

}  // namespace
}  // namespace evp

extern "C" int evp1d_run_device_noalloc(int na, int navel, const int32_t *ee,
                                        const int32_t *ne, const int32_t *se,
                                        const int32_t *nw, const int32_t *sw,
                                        const int32_t *sse, const double *dxT,
                                        const double *dyT, const double *HTE,
                                        const double *HTN, const double *HTEm1,
                                        const double *HTNm1, const double *uarear,
                                        const evp1d_params *params, int ndte,
                                        const evp1d_fields *io, void *stream) {
  using namespace evp;
  if (!params || !io) return error(EVP1D_ERR_INVALID_ARG, "params or io is NULL");
  if (na < 0 || navel < na || ndte < 0)
    return error(EVP1D_ERR_INVALID_ARG, "bad sizes na=%d navel=%d ndte=%d", na, navel,
                 ndte);
  if (navel > kNoAllocMaxNavel)
    return error(EVP1D_ERR_INVALID_ARG,
                 "navel %d exceeds the no-alloc scratch maximum %d "
                 "(EVP1D_NOALLOC_MAX_NAVEL); use evp1d_init/evp1d_run",
                 navel, kNoAllocMaxNavel);
  int dev = 0;
  NA_TRY(cudaGetDevice(&dev));
  double *scratch = nullptr;
  int *status = nullptr;
  int rc = scratch_in_context(&scratch, &status);
  if (rc != EVP1D_OK) return rc;
  if (na == 0 || ndte == 0) return EVP1D_OK;

  const void *must[] = {ee, ne, se, nw, sw, sse, dxT, dyT, HTE, HTN, HTEm1, HTNm1,
                        uarear, io->skipT, io->skipU, io->strength, io->Cw, io->aiu,
                        io->uocn, io->vocn, io->waterx, io->watery, io->forcex,
                        io->forcey, io->umassdti, io->fm, io->Tbu, io->uvel, io->vvel,
                        io->strintx, io->strinty, io->Cb};
  const char *names[] = {"ee", "ne", "se", "nw", "sw", "sse", "dxT", "dyT", "HTE",
                         "HTN", "HTEm1", "HTNm1", "uarear", "skipT", "skipU",
                         "strength", "Cw", "aiu", "uocn", "vocn", "waterx", "watery",
                         "forcex", "forcey", "umassdti", "fm", "Tbu", "uvel", "vvel",
                         "strintx", "strinty", "Cb"};
  for (size_t k = 0; k < sizeof must / sizeof must[0]; k++)
    if ((rc = check_device_ptr(must[k], dev, names[k])) != EVP1D_OK) return rc;
  for (int k = 0; k < 12; k++)
    if ((rc = check_device_ptr(io->stress[k], dev, "stress")) != EVP1D_OK) return rc;
  if ((io->uvel_init == nullptr) != (io->vvel_init == nullptr))
    return error(EVP1D_ERR_INVALID_ARG, "give both uvel_init and vvel_init or neither");
  if (io->uvel_init) {
    if ((rc = check_device_ptr(io->uvel_init, dev, "uvel_init")) != EVP1D_OK) return rc;
    if ((rc = check_device_ptr(io->vvel_init, dev, "vvel_init")) != EVP1D_OK) return rc;
  }
  for (int k = 0; k < 8; k++)
    if (io->str[k] && (rc = check_device_ptr(io->str[k], dev, "str")) != EVP1D_OK)
      return rc;

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  NaArgs a;
  a.na = na;
  a.navel = navel;
  a.ee = ee;
  a.ne = ne;
  a.se = se;
  a.nw = nw;
  a.sw = sw;
  a.sse = sse;
  a.skipT = io->skipT;
  a.skipU = io->skipU;
  a.dxT = dxT;
  a.dyT = dyT;
  a.HTE = HTE;
  a.HTN = HTN;
  a.HTEm1 = HTEm1;
  a.HTNm1 = HTNm1;
  a.uarear = uarear;
  a.strength = io->strength;
  a.Cw = io->Cw;
  a.aiu = io->aiu;
  a.uocn = io->uocn;
  a.vocn = io->vocn;
  a.waterx = io->waterx;
  a.watery = io->watery;
  a.forcex = io->forcex;
  a.forcey = io->forcey;
  a.umassdti = io->umassdti;
  a.fm = io->fm;
  a.Tbu = io->Tbu;
  for (int k = 0; k < 12; k++) a.stress[k] = io->stress[k];
  a.u = io->uvel;
  a.v = io->vvel;
  for (int k = 0; k < 8; k++) a.str[k] = scratch + k * (size_t)kNoAllocMaxNavel;
  a.strintx = io->strintx;
  a.strinty = io->strinty;
  a.Cb = io->Cb;
  if (io->uvel_init) {
    a.uinit = io->uvel_init;
    a.vinit = io->vvel_init;
  } else {
    double *ui = scratch + 8 * (size_t)kNoAllocMaxNavel;
    double *vi = scratch + 9 * (size_t)kNoAllocMaxNavel;
    NA_TRY(cudaMemcpyAsync(ui, io->uvel, sizeof(double) * na, cudaMemcpyDeviceToDevice, st));
    NA_TRY(cudaMemcpyAsync(vi, io->vvel, sizeof(double) * na, cudaMemcpyDeviceToDevice, st));
    a.uinit = ui;
    a.vinit = vi;
  }

  // neighbour check before any state is touched
  int host_status = kStatusNone;
  NA_TRY(cudaMemsetAsync(status, 0x7f, sizeof(int), st));
  k_na_check<<<grid_for(na), kThreads, 0, st>>>(a, status);
  NA_TRY(cudaGetLastError());
  NA_TRY(cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st));
  NA_TRY(cudaStreamSynchronize(st));
  if (host_status != kStatusNone)
    return error(EVP1D_ERR_INDEX,
                 "point %d (1-based) is the first with a neighbour outside 1..navel=%d",
                 host_status, navel);

  // str1..str8 start at zero on every call: stepu reads them at halo slots
  // and at skipped T points, which stress never writes.
  for (int k = 0; k < 8; k++)
    NA_TRY(cudaMemsetAsync(a.str[k], 0, sizeof(double) * navel, st));
  const int grid = grid_for(na);
  const Params p = kernel_params(*params);
  for (int s = 0; s < ndte; s++) {
    k_na_stress<<<grid, kThreads, 0, st>>>(a, p);
    k_na_stepu<<<grid, kThreads, 0, st>>>(a, p);
  }
  NA_TRY(cudaGetLastError());
  for (int k = 0; k < 8; k++)
    if (io->str[k])
      NA_TRY(cudaMemcpyAsync(io->str[k], a.str[k], sizeof(double) * navel,
                             cudaMemcpyDeviceToDevice, st));
  NA_TRY(cudaStreamSynchronize(st));
  return EVP1D_OK;
}
