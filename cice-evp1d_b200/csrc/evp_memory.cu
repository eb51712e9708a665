// evp_memory.cu -- device arena and host<->device movement of the 1D problem.
#include <cstring>
#include <vector>

#include "evp_internal.h"

namespace evp {

namespace {

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

#define CUDA_TRY(x)                                                        \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess)                                                 \
      return error(e_ == cudaErrorMemoryAllocation ? EVP1D_ERR_NOMEM       \
                                                   : EVP1D_ERR_CUDA,       \
                   "%s: %s", #x, cudaGetErrorString(e_));                  \
  } while (0)

int h2d(void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return EVP1D_OK;
  CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
  return EVP1D_OK;
}

int d2h(void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return EVP1D_OK;
  CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
  return EVP1D_OK;
}

}  // namespace

int internal_alloc(int device, int na, int navel, DevState *s, void **arena,
                   size_t *bytes, cudaStream_t *stream) {
  CUDA_TRY(cudaSetDevice(device));
  CUDA_TRY(cudaStreamCreateWithFlags(stream, cudaStreamNonBlocking));
  const size_t nA = (size_t)(na > 0 ? na : 1);
  const size_t nV = (size_t)(navel > 0 ? navel : 1);
  const size_t bi = align_up(nA * sizeof(int32_t));
  const size_t bf = align_up(nA);
  const size_t bd = align_up(nA * sizeof(double));
  const size_t bv = align_up(nV * sizeof(double));
  // 6 index vectors, flags, 7 geometry + 14 per-call + 12 stress + 3 output
  // fields of length na, u, v and str1..8 of length navel.
  const size_t total = 6 * bi + bf + (7 + 14 + 12 + 3) * bd + 10 * bv;
  void *base = nullptr;
  CUDA_TRY(cudaMalloc(&base, total));
  CUDA_TRY(cudaMemsetAsync(base, 0, total, *stream));
  char *p = (char *)base;
  auto take = [&](size_t b) {
    char *q = p;
    p += b;
    return q;
  };
  s->na = na;
  s->navel = navel;
  int32_t **idx[6] = {(int32_t **)&s->ee, (int32_t **)&s->ne,
                      (int32_t **)&s->se, (int32_t **)&s->nw,
                      (int32_t **)&s->sw, (int32_t **)&s->sse};
  for (int k = 0; k < 6; k++) *idx[k] = (int32_t *)take(bi);
  s->flags = (const uint8_t *)take(bf);
  const double **geo[7] = {&s->dxT, &s->dyT, &s->HTE, &s->HTN,
                           &s->HTEm1, &s->HTNm1, &s->uarear};
  for (int k = 0; k < 7; k++) *geo[k] = (const double *)take(bd);
  const double **dyn[14] = {&s->strength, &s->Cw, &s->aiu, &s->uocn,
                            &s->vocn, &s->waterx, &s->watery, &s->forcex,
                            &s->forcey, &s->umassdti, &s->fm, &s->Tbu,
                            &s->uinit, &s->vinit};
  for (int k = 0; k < 14; k++) *dyn[k] = (const double *)take(bd);
  for (int k = 0; k < 12; k++) s->stress[k] = (double *)take(bd);
  s->strintx = (double *)take(bd);
  s->strinty = (double *)take(bd);
  s->Cb = (double *)take(bd);
  s->u = (double *)take(bv);
  s->v = (double *)take(bv);
  for (int k = 0; k < 8; k++) s->str[k] = (double *)take(bv);
  *arena = base;
  *bytes = total;
  return EVP1D_OK;
}

int internal_upload_static(const DevState &s, const int32_t *const idx[6],
                           const double *const geo[7], cudaStream_t st) {
  const int na = s.na;
  if (na == 0) return EVP1D_OK;
  std::vector<int32_t> zb((size_t)na * 6);
  for (int k = 0; k < 6; k++)
    for (int w = 0; w < na; w++) zb[(size_t)k * na + w] = idx[k][w] - 1;
  const int32_t *dst[6] = {s.ee, s.ne, s.se, s.nw, s.sw, s.sse};
  for (int k = 0; k < 6; k++) {
    int rc = h2d((void *)dst[k], zb.data() + (size_t)k * na,
                 (size_t)na * sizeof(int32_t), st);
    if (rc) return rc;
  }
  const double *gdst[7] = {s.dxT, s.dyT, s.HTE, s.HTN, s.HTEm1, s.HTNm1,
                           s.uarear};
  for (int k = 0; k < 7; k++) {
    int rc = h2d((void *)gdst[k], geo[k], (size_t)na * sizeof(double), st);
    if (rc) return rc;
  }
  // the host staging vector dies here: wait for the copies.
  CUDA_TRY(cudaStreamSynchronize(st));
  return EVP1D_OK;
}

int internal_upload_fields(const DevState &s, const evp1d_fields *io,
                           std::vector<uint8_t> &flags_host, cudaStream_t st) {
  const int na = s.na, navel = s.navel;
  if (na == 0) return EVP1D_OK;
  const double *in[12] = {io->strength, io->Cw, io->aiu, io->uocn,
                          io->vocn, io->waterx, io->watery, io->forcex,
                          io->forcey, io->umassdti, io->fm, io->Tbu};
  static const char *inname[12] = {"strength", "Cw", "aiu", "uocn",
                                   "vocn", "waterx", "watery", "forcex",
                                   "forcey", "umassdti", "fm", "Tbu"};
  for (int k = 0; k < 12; k++)
    if (!in[k]) return error(EVP1D_ERR_INVALID_ARG, "field %s is NULL", inname[k]);
  for (int k = 0; k < 12; k++)
    if (!io->stress[k]) return error(EVP1D_ERR_INVALID_ARG, "stress[%d] is NULL", k);
  if (!io->skipT || !io->skipU || !io->uvel || !io->vvel || !io->strintx ||
      !io->strinty || !io->Cb)
    return error(EVP1D_ERR_INVALID_ARG,
                 "skipT/skipU/uvel/vvel/strintx/strinty/Cb must not be NULL");
  flags_host.resize((size_t)na);
  for (int w = 0; w < na; w++)
    flags_host[w] = (uint8_t)((io->skipT[w] ? kSkipT : 0) |
                              (io->skipU[w] ? kSkipU : 0));
  int rc = h2d((void *)s.flags, flags_host.data(), (size_t)na, st);
  if (rc) return rc;
  const double *dst[12] = {s.strength, s.Cw, s.aiu, s.uocn, s.vocn,
                           s.waterx, s.watery, s.forcex, s.forcey,
                           s.umassdti, s.fm, s.Tbu};
  const size_t bd = (size_t)na * sizeof(double);
  for (int k = 0; k < 12; k++)
    if ((rc = h2d((void *)dst[k], in[k], bd, st))) return rc;
  for (int k = 0; k < 12; k++)
    if ((rc = h2d(s.stress[k], io->stress[k], bd, st))) return rc;
  const size_t bv = (size_t)navel * sizeof(double);
  if ((rc = h2d(s.u, io->uvel, bv, st))) return rc;
  if ((rc = h2d(s.v, io->vvel, bv, st))) return rc;
  if (io->uvel_init) {
    if ((rc = h2d((void *)s.uinit, io->uvel_init, bd, st))) return rc;
  } else {
    CUDA_TRY(cudaMemcpyAsync((void *)s.uinit, s.u, bd, cudaMemcpyDeviceToDevice, st));
  }
  if (io->vvel_init) {
    if ((rc = h2d((void *)s.vinit, io->vvel_init, bd, st))) return rc;
  } else {
    CUDA_TRY(cudaMemcpyAsync((void *)s.vinit, s.v, bd, cudaMemcpyDeviceToDevice, st));
  }
  if ((rc = h2d(s.strintx, io->strintx, bd, st))) return rc;
  if ((rc = h2d(s.strinty, io->strinty, bd, st))) return rc;
  if ((rc = h2d(s.Cb, io->Cb, bd, st))) return rc;
  for (int k = 0; k < 8; k++) CUDA_TRY(cudaMemsetAsync(s.str[k], 0, bv, st));
  // flags_host must stay alive until its copy has run.
  CUDA_TRY(cudaStreamSynchronize(st));
  return EVP1D_OK;
}

int internal_download_fields(const DevState &s, const evp1d_fields *io,
                             cudaStream_t st) {
  const int na = s.na, navel = s.navel;
  if (na == 0) return EVP1D_OK;
  const size_t bd = (size_t)na * sizeof(double);
  const size_t bv = (size_t)navel * sizeof(double);
  int rc;
  for (int k = 0; k < 12; k++)
    if (io->stress[k] && (rc = d2h(io->stress[k], s.stress[k], bd, st))) return rc;
  if (io->uvel && (rc = d2h(io->uvel, s.u, bd, st))) return rc;
  if (io->vvel && (rc = d2h(io->vvel, s.v, bd, st))) return rc;
  if (io->strintx && (rc = d2h(io->strintx, s.strintx, bd, st))) return rc;
  if (io->strinty && (rc = d2h(io->strinty, s.strinty, bd, st))) return rc;
  if (io->Cb && (rc = d2h(io->Cb, s.Cb, bd, st))) return rc;
  for (int k = 0; k < 8; k++)
    if (io->str[k] && (rc = d2h(io->str[k], s.str[k], bv, st))) return rc;
  CUDA_TRY(cudaStreamSynchronize(st));
  return EVP1D_OK;
}

}  // namespace evp
