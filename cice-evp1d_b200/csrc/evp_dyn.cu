// evp_dyn.cu -- the 2D adapter of include/evp1d.h (evp1d_dyn_*): the
// dyn_evp1d_init / dyn_evp1d_run / dyn_evp1d_finalize interface on global 2D
// arrays, on top of the 1D solver.
//
// The per-timestep conversions run on the device: the caller's 2D arrays are
// copied whole to the GPU, a gather kernel builds the 1D list fields and the
// skip flags (convert_2d_1d_dyn and set_skipMe,
// integration/ice_dyn_evp1d.F90:521-537, 818-882) straight into the solver's
// staging area, and after the subcycles a scatter kernel writes the list
// points' results back into the 2D arrays (convert_1d_2d_dyn, :884-947),
// which are copied back whole.  Cells outside the list keep the values the
// caller passed.
#include <cstdint>
#include <string>
#include <vector>

#include "evp1d.h"
#include "evp_handle.h"
#include "evp_internal.h"

namespace {

// 2D fields of one call on the device, in this order: the 12 per-call inputs
// (strength, cdn_ocn, aiu, uocn, vocn, waterxU, wateryU, forcexU, forceyU,
// umassdti, fmU, Tbu), the 12 stresses, strintxU, strintyU, Cb, uvel, vvel.
constexpr int kIn2d = 12;
constexpr int kF2d = kIn2d + 12 + 3 + 2;  // 29
constexpr int kOut2d = 12 + 3 + 2;        // results: stresses, strint, Cb, u, v

struct Gather2d {
  const double *f[kF2d];
  const int32_t *icet, *iceu;
};

// 2D -> reference-order staging (slots of problem_upload_staged): list points
// from their cells, halo slots of u and v zero (:880-881), skip flags from the
// ice masks (set_skipMe).
__global__ void k_gather_2d(int na, int navel, const int32_t *__restrict__ cell, Gather2d g,
                            double *stage) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < navel;
       p += gridDim.x * blockDim.x) {
    auto slot = [&](int k) { return stage + (size_t)k * navel; };
    if (p >= na) {
      slot(24)[p] = 0.0;
      slot(25)[p] = 0.0;
      continue;
    }
    const int c = cell[p];
#pragma unroll
    for (int k = 0; k < kIn2d; k++) slot(k)[p] = g.f[k][c];
#pragma unroll
    for (int k = 0; k < 12; k++) slot(12 + k)[p] = g.f[kIn2d + k][c];
    slot(28)[p] = g.f[24][c];
    slot(29)[p] = g.f[25][c];
    slot(30)[p] = g.f[26][c];
    slot(24)[p] = g.f[27][c];
    slot(25)[p] = g.f[28][c];
    int32_t *skT = reinterpret_cast<int32_t *>(slot(31));
    skT[p] = g.icet[c] ? 0 : 1;
    skT[navel + p] = g.iceu[c] ? 0 : 1;
  }
}

struct Scatter2d {
  double *f[kOut2d];
};

// Reference-order results (slots of problem_download_staged) -> their cells.
__global__ void k_scatter_2d(int na, int navel, const int32_t *__restrict__ cell,
                             const double *stage, Scatter2d o) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < na; p += gridDim.x * blockDim.x) {
    const int c = cell[p];
#pragma unroll
    for (int k = 0; k < 12; k++) o.f[k][c] = stage[(size_t)k * navel + p];
    o.f[12][c] = stage[(size_t)14 * navel + p];  // strintx
    o.f[13][c] = stage[(size_t)15 * navel + p];  // strinty
    o.f[14][c] = stage[(size_t)16 * navel + p];  // Cb
    o.f[15][c] = stage[(size_t)12 * navel + p];  // uvel
    o.f[16][c] = stage[(size_t)13 * navel + p];  // vvel
  }
}

int grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148LL * 32) b = 148LL * 32;
  return (int)b;
}

#define DYN_TRY(x)                                                         \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess)                                                 \
      return evp::error(e_ == cudaErrorMemoryAllocation ? EVP1D_ERR_NOMEM  \
                                                       : EVP1D_ERR_CUDA,   \
                        "%s: %s", #x, cudaGetErrorString(e_));             \
  } while (0)

}  // namespace

struct evp1d_dyn_handle {
  int nx = 0, ny = 0, na = 0, navel = 0;
  evp1d_t *h = nullptr;
  int32_t *cell = nullptr;   // device: 2D cell (0-based, i fastest) of each list point
  double *f2d = nullptr;     // device: kF2d x nx*ny doubles
  int32_t *mask2d = nullptr; // device: icetmask, iceumask
};

extern "C" {

int evp1d_dyn_init(evp1d_dyn_t **handle, int nx, int ny, int nghost,
                   const int32_t *tmask, const double *dyT, const double *dxT,
                   const double *uarear, const double *HTE, const double *HTN,
                   const evp1d_params *params, int device) {
  if (!handle || !tmask || !dyT || !dxT || !uarear || !HTE || !HTN || !params)
    return evp::error(EVP1D_ERR_INVALID_ARG, "NULL argument");
  *handle = nullptr;
  if (nx < 2 || ny < 2 || nghost < 1)
    return evp::error(EVP1D_ERR_INVALID_ARG, "need nx, ny >= 2 and nghost >= 1");
  if ((long long)nx * ny > 0x7fffffffLL)
    return evp::error(EVP1D_ERR_INVALID_ARG, "nx*ny too large for int32 cell indices");
  int na = 0, navel = 0;
  int rc = evp1d_build_index(nx, ny, nghost, tmask, 0, 0, &na, &navel, nullptr, nullptr,
                             nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (rc != EVP1D_OK && rc != EVP1D_ERR_INVALID_ARG) return rc;
  std::vector<int32_t> ti((size_t)na + 1), tj((size_t)na + 1), tij((size_t)navel + 1),
      nb((size_t)6 * (na + 1));
  int32_t *nbp[6];
  for (int k = 0; k < 6; k++) nbp[k] = nb.data() + (size_t)k * (na + 1);
  rc = evp1d_build_index(nx, ny, nghost, tmask, na, navel, &na, &navel, ti.data(), tj.data(),
                         tij.data(), nbp[0], nbp[1], nbp[2], nbp[3], nbp[4], nbp[5]);
  if (rc != EVP1D_OK) return rc;
  // static 1D geometry (convert_2d_1d_init, :803-815): HTEm1 = HTE(i-1,j),
  // HTNm1 = HTN(i,j-1)
  std::vector<int32_t> cell((size_t)na + 1);
  std::vector<double> g((size_t)7 * (na + 1));
  double *G[7];
  for (int k = 0; k < 7; k++) G[k] = g.data() + (size_t)k * (na + 1);
  for (int w = 0; w < na; w++) {
    const size_t c = (size_t)(ti[w] - 1) + (size_t)(tj[w] - 1) * (size_t)nx;
    cell[w] = (int32_t)c;
    G[0][w] = dxT[c];
    G[1][w] = dyT[c];
    G[2][w] = HTE[c];
    G[3][w] = HTN[c];
    G[4][w] = HTE[c - 1];
    G[5][w] = HTN[c - (size_t)nx];
    G[6][w] = uarear[c];
  }
  evp1d_dyn_t *d = new evp1d_dyn_handle();
  d->nx = nx;
  d->ny = ny;
  d->na = na;
  d->navel = navel;
  rc = evp1d_init(&d->h, na, navel, nbp[0], nbp[1], nbp[2], nbp[3], nbp[4], nbp[5], G[0],
                  G[1], G[2], G[3], G[4], G[5], G[6], params, device);
  if (rc != EVP1D_OK) {
    delete d;
    return rc;
  }
  if (na > 0) {
    const size_t cells = (size_t)nx * ny;
    cudaError_t e = evp::device_alloc(&d->cell, sizeof(int32_t) * (size_t)na);
    if (e == cudaSuccess) e = evp::device_alloc(&d->f2d, sizeof(double) * kF2d * cells);
    if (e == cudaSuccess) e = evp::device_alloc(&d->mask2d, sizeof(int32_t) * 2 * cells);
    if (e == cudaSuccess)
      e = cudaMemcpy(d->cell, cell.data(), sizeof(int32_t) * (size_t)na, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      evp1d_dyn_finalize(d);
      return evp::error(e == cudaErrorMemoryAllocation ? EVP1D_ERR_NOMEM : EVP1D_ERR_CUDA,
                        "2D adapter buffers: %s", cudaGetErrorString(e));
    }
  }
  *handle = d;
  return EVP1D_OK;
}

int evp1d_dyn_run(evp1d_dyn_t *d, int ndte, const evp1d_dyn_fields *io) {
  evp::NvtxRange nvtx_range("evp1d_dyn_run");
  if (!d || !io) return evp::error(EVP1D_ERR_INVALID_ARG, "NULL argument");
  const double *in[kIn2d] = {io->strength, io->cdn_ocn, io->aiu, io->uocn, io->vocn,
                             io->waterxU, io->wateryU, io->forcexU, io->forceyU,
                             io->umassdti, io->fmU, io->Tbu};
  for (int k = 0; k < kIn2d; k++)
    if (!in[k] || !io->stress[k]) return evp::error(EVP1D_ERR_INVALID_ARG, "NULL field");
  if (!io->strintxU || !io->strintyU || !io->Cb || !io->uvel || !io->vvel ||
      !io->icetmask || !io->iceumask)
    return evp::error(EVP1D_ERR_INVALID_ARG, "NULL field");
  if (ndte < 0) return evp::error(EVP1D_ERR_INVALID_ARG, "ndte = %d < 0", ndte);
  if (d->na == 0) return EVP1D_OK;
  evp1d_t *h = d->h;
  evp::DeviceProblem &P = h->d;
  DYN_TRY(cudaSetDevice(P.device));
  cudaStream_t st = P.stream;
  const size_t cells = (size_t)d->nx * d->ny, bc = sizeof(double) * cells;
  // whole 2D arrays to the device
  const double *src[kF2d];
  for (int k = 0; k < kIn2d; k++) src[k] = in[k];
  for (int k = 0; k < 12; k++) src[kIn2d + k] = io->stress[k];
  src[24] = io->strintxU;
  src[25] = io->strintyU;
  src[26] = io->Cb;
  src[27] = io->uvel;
  src[28] = io->vvel;
  Gather2d g;
  for (int k = 0; k < kF2d; k++) {
    double *dst = d->f2d + (size_t)k * cells;
    DYN_TRY(cudaMemcpyAsync(dst, src[k], bc, cudaMemcpyHostToDevice, st));
    g.f[k] = dst;
  }
  DYN_TRY(cudaMemcpyAsync(d->mask2d, io->icetmask, sizeof(int32_t) * cells,
                          cudaMemcpyHostToDevice, st));
  DYN_TRY(cudaMemcpyAsync(d->mask2d + cells, io->iceumask, sizeof(int32_t) * cells,
                          cudaMemcpyHostToDevice, st));
  g.icet = d->mask2d;
  g.iceu = d->mask2d + cells;
  // 2D -> 1D staging on the device, then the solver's own upload
  k_gather_2d<<<grid_for(d->navel), 256, 0, st>>>(d->na, d->navel, d->cell, g, P.stage);
  DYN_TRY(cudaGetLastError());
  evp::adjoint_invalidate(h->adj);
  h->uinit_explicit = false;
  int rc = evp::problem_upload_staged(&P, false, false, h->p.rhow);
  if (rc != EVP1D_OK) return rc;
  h->uploaded = true;
  rc = evp1d_subcycles(h, ndte);
  if (rc != EVP1D_OK) return rc;
  rc = evp1d_synchronize(h);  // also reports a bounded device wait that ran out
  if (rc != EVP1D_OK) return rc;
  // 1D results -> their cells of the device copies -> the caller's arrays
  const bool no_str[8] = {false, false, false, false, false, false, false, false};
  rc = evp::problem_download_staged(&P, no_str);
  if (rc != EVP1D_OK) return rc;
  Scatter2d o;
  double *dst[kOut2d];
  for (int k = 0; k < 12; k++) o.f[k] = d->f2d + (size_t)(kIn2d + k) * cells;
  for (int k = 0; k < 5; k++) o.f[12 + k] = d->f2d + (size_t)(24 + k) * cells;
  k_scatter_2d<<<grid_for(d->na), 256, 0, st>>>(d->na, d->navel, d->cell, P.stage, o);
  DYN_TRY(cudaGetLastError());
  for (int k = 0; k < 12; k++) dst[k] = io->stress[k];
  dst[12] = io->strintxU;
  dst[13] = io->strintyU;
  dst[14] = io->Cb;
  dst[15] = io->uvel;
  dst[16] = io->vvel;
  for (int k = 0; k < kOut2d; k++)
    DYN_TRY(cudaMemcpyAsync(dst[k], o.f[k], bc, cudaMemcpyDeviceToHost, st));
  DYN_TRY(cudaStreamSynchronize(st));
  return EVP1D_OK;
}

int evp1d_dyn_finalize(evp1d_dyn_t *d) {
  if (!d) return EVP1D_OK;
  int rc = EVP1D_OK;
  if (d->h) {
    cudaSetDevice(d->h->d.device);
    if (d->cell) cudaFree(d->cell);
    if (d->f2d) cudaFree(d->f2d);
    if (d->mask2d) cudaFree(d->mask2d);
    rc = evp1d_finalize(d->h);
  }
  delete d;
  return rc;
}

int evp1d_dyn_sizes(evp1d_dyn_t *d, int *na, int *navel) {
  if (!d || !na || !navel) return evp::error(EVP1D_ERR_INVALID_ARG, "NULL argument");
  *na = d->na;
  *navel = d->navel;
  return EVP1D_OK;
}

}  // extern "C"
