// evp_problem.cu -- device arena of one 1D problem and its movement between
// the caller's reference-order host arrays and the slot-ordered device state.
#include <cstring>
#include <vector>

#include "evp_internal.h"

namespace evp {

namespace {

#define CUDA_TRY(x)                                                        \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess)                                                 \
      return error(e_ == cudaErrorMemoryAllocation ? EVP1D_ERR_NOMEM       \
                                                   : EVP1D_ERR_CUDA,       \
                   "%s: %s", #x, cudaGetErrorString(e_));                  \
  } while (0)

#define TRY(x)               \
  do {                       \
    int rc_ = (x);           \
    if (rc_) return rc_;     \
  } while (0)

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// Bump allocator over one cudaMalloc.
struct Carve {
  char *base = nullptr;
  size_t off = 0;
  template <class T>
  void take(T **p, size_t count) {
    const size_t b = align_up((count > 0 ? count : 1) * sizeof(T));
    if (base) *p = (T *)(base + off);
    off += b;
  }
};

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

void layout(DeviceProblem *d, Carve &c, size_t nhalo_total, size_t nuvx_total,
            size_t ndep_total) {
  const size_t S = (size_t)d->nslots, U = (size_t)d->nuv, T = (size_t)d->ntiles;
  c.take(&d->err, 1);
  c.take(&d->cflags, 1);
  c.take(&d->meta, S);
  c.take(&d->lcor, S);
  c.take(&d->halo_lcc, nhalo_total);
  c.take(&d->halo_lcor, nhalo_total);
  c.take(&d->uvx_off, T);
  c.take(&d->uvx_cnt, T);
  c.take(&d->uvx_idx, nuvx_total);
  c.take(&d->tile_meta, 8 * T);
  c.take(&d->tile_rec, (size_t)kRecInts * T);
  c.take(&d->cblk, (size_t)kConstFields * kConstTileSlots * T);
  c.take(&d->run_off, (size_t)d->nruns + 1);
  c.take(&d->dep_off, T + 1);
  c.take(&d->dep_idx, ndep_total);
  c.take(&d->epoch, T);
  c.take(&d->tile_off, T);
  c.take(&d->tile_cnt, T);
  c.take(&d->halo_off, T);
  c.take(&d->halo_cnt, T);
  c.take(&d->halo_idx, nhalo_total);
  c.take(&d->slot_of_point, (size_t)d->na);
  c.take(&d->point_of_slot, S);
  for (int k = 0; k < 6; k++) c.take(&d->nb[k], S);
  c.take(&d->lnb, S);
  c.take(&d->flags, S);
  for (int k = 0; k < kNumGeo; k++) c.take(&d->geo[k], S);
  for (int k = 0; k < kNumDyn; k++) c.take(&d->dyn[k], S);
  for (int b = 0; b < 2; b++) {
    for (int k = 0; k < 12; k++) c.take(&d->stress[b][k], S);
    c.take(&d->u[b], U);
    c.take(&d->v[b], U);
  }
  c.take(&d->strintx, S);
  c.take(&d->strinty, S);
  c.take(&d->Cb, S);
  for (int k = 0; k < 8; k++) c.take(&d->str[k], U);
  c.take(&d->stage, (size_t)32 * (size_t)(d->navel > 0 ? d->navel : 1));
}

}  // namespace

int problem_create(DeviceProblem *d, int device, const TilePlan &plan,
                   const double *const geo[kNumGeo]) {
  d->device = device;
  d->na = plan.na;
  d->navel = plan.navel;
  d->nslots = plan.nslots;
  d->nhs = plan.nhalo_slots;
  d->nuv = plan.nslots + plan.nhalo_slots;
  d->ntiles = plan.ntiles;
  d->nruns = plan.nruns;
  d->from_coords = plan.from_coords;
  CUDA_TRY(cudaSetDevice(device));
  CUDA_TRY(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking));
  CUDA_TRY(cudaDeviceGetAttribute(&d->nctas, cudaDevAttrMultiProcessorCount, device));
  if (tma_prepare(device) != 0)
    return error(EVP1D_ERR_CUDA, "cannot enable %d bytes of shared memory", 0);
  Carve sizing;
  layout(d, sizing, plan.halo_idx.size(), plan.uvx_idx.size(), plan.dep_idx.size());
  CUDA_TRY(device_alloc(&d->arena, sizing.off));
  d->arena_bytes = sizing.off;
  Carve c;
  c.base = (char *)d->arena;
  layout(d, c, plan.halo_idx.size(), plan.uvx_idx.size(), plan.dep_idx.size());
  cudaStream_t st = d->stream;
  CUDA_TRY(cudaMemsetAsync(d->arena, 0, d->arena_bytes, st));
  if (d->na == 0) {
    CUDA_TRY(cudaStreamSynchronize(st));
    return EVP1D_OK;
  }
  const size_t T = (size_t)d->ntiles * sizeof(int32_t);
  const size_t S4 = (size_t)d->nslots * sizeof(int32_t);
  TRY(h2d(d->run_off, plan.run_off.data(), plan.run_off.size() * sizeof(int32_t), st));
  TRY(h2d(d->dep_off, plan.dep_off.data(), plan.dep_off.size() * sizeof(int32_t), st));
  TRY(h2d(d->dep_idx, plan.dep_idx.data(), plan.dep_idx.size() * sizeof(int32_t), st));
  TRY(h2d(d->tile_off, plan.tile_off.data(), T, st));
  TRY(h2d(d->tile_cnt, plan.tile_cnt.data(), T, st));
  TRY(h2d(d->halo_off, plan.halo_off.data(), T, st));
  TRY(h2d(d->halo_cnt, plan.halo_cnt.data(), T, st));
  TRY(h2d(d->halo_idx, plan.halo_idx.data(), plan.halo_idx.size() * sizeof(int32_t), st));
  TRY(h2d(d->slot_of_point, plan.slot_of_point.data(), (size_t)d->na * sizeof(int32_t), st));
  TRY(h2d(d->point_of_slot, plan.point_of_slot.data(), S4, st));
  const std::vector<int32_t> *nbv[6] = {&plan.ee, &plan.ne, &plan.se,
                                        &plan.nw, &plan.sw, &plan.sse};
  for (int k = 0; k < 6; k++) TRY(h2d(d->nb[k], nbv[k]->data(), S4, st));
  TRY(h2d(d->lnb, plan.lnb.data(), S4, st));
  TRY(h2d(d->meta, plan.lnb.data(), S4, st));
  TRY(h2d(d->lcor, plan.lcor.data(), S4, st));
  const size_t H4 = plan.halo_idx.size() * sizeof(uint32_t);
  TRY(h2d(d->halo_lcc, plan.halo_lcc.data(), H4, st));
  TRY(h2d(d->halo_lcor, plan.halo_lcor.data(), H4, st));
  TRY(h2d(d->uvx_off, plan.uvx_off.data(), T, st));
  TRY(h2d(d->uvx_cnt, plan.uvx_cnt.data(), T, st));
  TRY(h2d(d->uvx_idx, plan.uvx_idx.data(), plan.uvx_idx.size() * sizeof(int32_t), st));
  std::vector<int32_t> tm((size_t)8 * d->ntiles, 0);
  for (int t = 0; t < d->ntiles; t++) {
    int32_t *q = tm.data() + (size_t)8 * t;
    q[0] = plan.tile_off[t];
    q[1] = plan.tile_cnt[t];
    q[2] = plan.uvx_off[t];
    q[3] = plan.uvx_cnt[t];
    q[4] = plan.halo_off[t];
    q[5] = plan.halo_cnt[t];
  }
  TRY(h2d(d->tile_meta, tm.data(), tm.size() * sizeof(int32_t), st));
  std::vector<int32_t> rec((size_t)kRecInts * d->ntiles, 0);
  for (int t = 0; t < d->ntiles; t++) {
    int32_t *q = rec.data() + (size_t)kRecInts * t;
    const int nx = plan.uvx_cnt[t], nh = plan.halo_cnt[t];
    q[0] = plan.tile_off[t];
    q[1] = plan.tile_cnt[t];
    q[2] = nx;
    q[3] = nh;
    for (int x = 0; x < nx; x++) q[kRecUvx + x] = plan.uvx_idx[plan.uvx_off[t] + x];
    for (int h = 0; h < nh; h++) {
      q[kRecHalo + h] = plan.halo_idx[plan.halo_off[t] + h];
      q[kRecHLcor + h] = (int32_t)plan.halo_lcor[plan.halo_off[t] + h];
      q[kRecHLcc + h] = (int32_t)plan.halo_lcc[plan.halo_off[t] + h];
    }
  }
  TRY(h2d(d->tile_rec, rec.data(), rec.size() * sizeof(int32_t), st));
  // geometry: reference order -> staging -> slots
  PermBatch b;
  for (int k = 0; k < kNumGeo; k++) {
    double *src = d->stage + (size_t)k * d->navel;
    TRY(h2d(src, geo[k], (size_t)d->na * sizeof(double), st));
    b.src[b.n] = src;
    b.dst[b.n] = d->geo[k];
    b.n++;
  }
  launch_scatter(b, d->nslots, d->point_of_slot, st);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(st));
  return EVP1D_OK;
}

void problem_destroy(DeviceProblem *d) {
  if (d->stream) {
    cudaSetDevice(d->device);
    cudaStreamSynchronize(d->stream);
  }
  if (d->arena) cudaFree(d->arena);
  if (d->stream) cudaStreamDestroy(d->stream);
  d->arena = nullptr;
  d->stream = nullptr;
}

int problem_upload(DeviceProblem *d, const evp1d_fields *io, double rhow) {
  const int na = d->na, navel = d->navel;
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
  cudaStream_t st = d->stream;
  const size_t bd = (size_t)na * sizeof(double);
  const size_t bv = (size_t)navel * sizeof(double);
  auto slot = [&](int k) { return d->stage + (size_t)k * navel; };
  // staging slots: 0..11 per-call inputs, 12..23 stresses, 24 u, 25 v,
  // 26 uinit, 27 vinit, 28 strintx, 29 strinty, 30 Cb, 31 skipT|skipU (int32)
  for (int k = 0; k < 12; k++) TRY(h2d(slot(k), in[k], bd, st));
  for (int k = 0; k < 12; k++) TRY(h2d(slot(12 + k), io->stress[k], bd, st));
  TRY(h2d(slot(24), io->uvel, bv, st));
  TRY(h2d(slot(25), io->vvel, bv, st));
  if (io->uvel_init) TRY(h2d(slot(26), io->uvel_init, bd, st));
  if (io->vvel_init) TRY(h2d(slot(27), io->vvel_init, bd, st));
  TRY(h2d(slot(28), io->strintx, bd, st));
  TRY(h2d(slot(29), io->strinty, bd, st));
  TRY(h2d(slot(30), io->Cb, bd, st));
  int32_t *skT = (int32_t *)slot(31);
  int32_t *skU = skT + navel;  // 2 x navel int32 fit in navel doubles
  TRY(h2d(skT, io->skipT, (size_t)na * sizeof(int32_t), st));
  TRY(h2d(skU, io->skipU, (size_t)na * sizeof(int32_t), st));
  return problem_upload_staged(d, io->uvel_init != nullptr, io->vvel_init != nullptr, rhow);
}

int problem_upload_staged(DeviceProblem *d, bool uinit_given, bool vinit_given, double rhow) {
  const int na = d->na, navel = d->navel;
  if (na == 0) return EVP1D_OK;
  cudaStream_t st = d->stream;
  auto slot = [&](int k) { return d->stage + (size_t)k * navel; };
  const double *uinit_src = uinit_given ? slot(26) : slot(24);
  const double *vinit_src = vinit_given ? slot(27) : slot(25);
  int32_t *skT = (int32_t *)slot(31);
  int32_t *skU = skT + navel;
  launch_flags(d->nslots, d->point_of_slot, skT, skU, d->flags, d->lnb, d->meta, st);
  PermBatch a;  // single-copy fields
  for (int k = 0; k < 12; k++) {
    a.src[a.n] = slot(k);
    a.dst[a.n++] = d->dyn[k];
  }
  a.src[a.n] = uinit_src;
  a.dst[a.n++] = d->dyn[kUinit];
  a.src[a.n] = vinit_src;
  a.dst[a.n++] = d->dyn[kVinit];
  a.src[a.n] = slot(28);
  a.dst[a.n++] = d->strintx;
  a.src[a.n] = slot(29);
  a.dst[a.n++] = d->strinty;
  a.src[a.n] = slot(30);
  a.dst[a.n++] = d->Cb;
  launch_scatter(a, d->nslots, d->point_of_slot, st);
  PermBatch b;  // state: both ping-pong buffers
  for (int k = 0; k < 12; k++) {
    b.src[b.n] = slot(12 + k);
    b.dst[b.n] = d->stress[0][k];
    b.dst2[b.n++] = d->stress[1][k];
  }
  b.src[b.n] = slot(24);
  b.dst[b.n] = d->u[0];
  b.dst2[b.n++] = d->u[1];
  b.src[b.n] = slot(25);
  b.dst[b.n] = d->v[0];
  b.dst2[b.n++] = d->v[1];
  launch_scatter(b, d->nslots, d->point_of_slot, st);
  CUDA_TRY(cudaGetLastError());
  if (d->nhs > 0) {
    const size_t bh = (size_t)d->nhs * sizeof(double);
    for (int k = 0; k < 2; k++) {
      CUDA_TRY(cudaMemcpyAsync(d->u[k] + d->nslots, slot(24) + na, bh,
                               cudaMemcpyDeviceToDevice, st));
      CUDA_TRY(cudaMemcpyAsync(d->v[k] + d->nslots, slot(25) + na, bh,
                               cudaMemcpyDeviceToDevice, st));
    }
  }
  launch_drag_factor(d->nslots, d->dyn[kAiu], d->dyn[kCw], rhow, d->dyn[kKvrel], st);
  TRY(problem_fill_const(d));
  for (int k = 0; k < 8; k++)
    CUDA_TRY(cudaMemsetAsync(d->str[k], 0, (size_t)d->nuv * sizeof(double), st));
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(st));
  d->cur = 0;
  return EVP1D_OK;
}

int problem_fill_const(DeviceProblem *d) {
  if (d->ntiles == 0) return EVP1D_OK;
  const double *src[kConstFields - 1] = {
      d->geo[kDxT],  d->geo[kDyT],    d->geo[kHTE],    d->geo[kHTN],    d->geo[kHTEm1],
      d->geo[kHTNm1], d->dyn[kStrength], d->dyn[kKvrel], d->dyn[kUocn], d->dyn[kVocn],
      d->dyn[kWaterx], d->dyn[kWatery], d->dyn[kForcex], d->dyn[kForcey], d->dyn[kUmassdti],
      d->dyn[kFm],   d->geo[kUarear], d->dyn[kTbu],    d->dyn[kUinit],  d->dyn[kVinit]};
  CUDA_TRY(cudaMemsetAsync(d->cflags, 0, sizeof(int), d->stream));
  launch_const_blocks(d->ntiles, d->tile_off, d->tile_cnt, src, d->meta, d->lcor, d->cblk,
                      d->cflags, d->stream);
  CUDA_TRY(cudaGetLastError());
  return EVP1D_OK;
}

int problem_download(DeviceProblem *d, const evp1d_fields *io) {
  const int na = d->na, navel = d->navel;
  if (na == 0) return EVP1D_OK;
  cudaStream_t st = d->stream;
  auto slot = [&](int k) { return d->stage + (size_t)k * navel; };
  bool want_str[8];
  for (int k = 0; k < 8; k++) want_str[k] = io->str[k] != nullptr;
  TRY(problem_download_staged(d, want_str));
  const size_t bd = (size_t)na * sizeof(double);
  for (int k = 0; k < 12; k++)
    if (io->stress[k]) TRY(d2h(io->stress[k], slot(k), bd, st));
  if (io->uvel) TRY(d2h(io->uvel, slot(12), bd, st));
  if (io->vvel) TRY(d2h(io->vvel, slot(13), bd, st));
  if (io->strintx) TRY(d2h(io->strintx, slot(14), bd, st));
  if (io->strinty) TRY(d2h(io->strinty, slot(15), bd, st));
  if (io->Cb) TRY(d2h(io->Cb, slot(16), bd, st));
  for (int k = 0; k < 8; k++)
    if (io->str[k]) {
      TRY(d2h(io->str[k], slot(17 + k), bd, st));
      if (d->nhs > 0)
        TRY(d2h(io->str[k] + na, d->str[k] + d->nslots,
                (size_t)d->nhs * sizeof(double), st));
    }
  CUDA_TRY(cudaStreamSynchronize(st));
  return EVP1D_OK;
}

int problem_download_staged(DeviceProblem *d, const bool want_str[8]) {
  const int na = d->na, navel = d->navel;
  if (na == 0) return EVP1D_OK;
  cudaStream_t st = d->stream;
  auto slot = [&](int k) { return d->stage + (size_t)k * navel; };
  PermBatch g;
  const int c = d->cur;
  for (int k = 0; k < 12; k++) {
    g.src[g.n] = d->stress[c][k];
    g.dst[g.n++] = slot(k);
  }
  g.src[g.n] = d->u[c];
  g.dst[g.n++] = slot(12);
  g.src[g.n] = d->v[c];
  g.dst[g.n++] = slot(13);
  g.src[g.n] = d->strintx;
  g.dst[g.n++] = slot(14);
  g.src[g.n] = d->strinty;
  g.dst[g.n++] = slot(15);
  g.src[g.n] = d->Cb;
  g.dst[g.n++] = slot(16);
  for (int k = 0; k < 8; k++)
    if (want_str[k]) {
      g.src[g.n] = d->str[k];
      g.dst[g.n++] = slot(17 + k);
    }
  launch_gather(g, na, d->slot_of_point, st);
  CUDA_TRY(cudaGetLastError());
  return EVP1D_OK;
}

DevState problem_inplace_view(const DeviceProblem &d) {
  DevState s;
  const int c = d.cur;
  s.na = d.nslots;
  s.navel = d.nuv;
  s.ee = d.nb[0];
  s.ne = d.nb[1];
  s.se = d.nb[2];
  s.nw = d.nb[3];
  s.sw = d.nb[4];
  s.sse = d.nb[5];
  s.flags = d.flags;
  s.dxT = d.geo[kDxT];
  s.dyT = d.geo[kDyT];
  s.HTE = d.geo[kHTE];
  s.HTN = d.geo[kHTN];
  s.HTEm1 = d.geo[kHTEm1];
  s.HTNm1 = d.geo[kHTNm1];
  s.uarear = d.geo[kUarear];
  s.strength = d.dyn[kStrength];
  s.Cw = d.dyn[kCw];
  s.aiu = d.dyn[kAiu];
  s.uocn = d.dyn[kUocn];
  s.vocn = d.dyn[kVocn];
  s.waterx = d.dyn[kWaterx];
  s.watery = d.dyn[kWatery];
  s.forcex = d.dyn[kForcex];
  s.forcey = d.dyn[kForcey];
  s.umassdti = d.dyn[kUmassdti];
  s.fm = d.dyn[kFm];
  s.Tbu = d.dyn[kTbu];
  s.uinit = d.dyn[kUinit];
  s.vinit = d.dyn[kVinit];
  for (int k = 0; k < 12; k++) s.stress[k] = d.stress[c][k];
  s.u = d.u[c];
  s.v = d.v[c];
  for (int k = 0; k < 8; k++) s.str[k] = d.str[k];
  s.strintx = d.strintx;
  s.strinty = d.strinty;
  s.Cb = d.Cb;
  return s;
}

FusedArgs problem_fused_args(const DeviceProblem &d, int from) {
  FusedArgs a;
  const int to = 1 - from;
  a.ntiles = d.ntiles;
  a.nruns = d.nruns;
  a.run_off = d.run_off;
  a.tile_off = d.tile_off;
  a.tile_cnt = d.tile_cnt;
  a.halo_off = d.halo_off;
  a.halo_cnt = d.halo_cnt;
  a.halo_idx = d.halo_idx;
  a.flags = d.flags;
  a.ee = d.nb[0];
  a.ne = d.nb[1];
  a.se = d.nb[2];
  a.lnb = d.lnb;
  a.dxT = d.geo[kDxT];
  a.dyT = d.geo[kDyT];
  a.HTE = d.geo[kHTE];
  a.HTN = d.geo[kHTN];
  a.HTEm1 = d.geo[kHTEm1];
  a.HTNm1 = d.geo[kHTNm1];
  a.uarear = d.geo[kUarear];
  a.strength = d.dyn[kStrength];
  a.kvrel = d.dyn[kKvrel];
  a.uocn = d.dyn[kUocn];
  a.vocn = d.dyn[kVocn];
  a.waterx = d.dyn[kWaterx];
  a.watery = d.dyn[kWatery];
  a.forcex = d.dyn[kForcex];
  a.forcey = d.dyn[kForcey];
  a.umassdti = d.dyn[kUmassdti];
  a.fm = d.dyn[kFm];
  a.Tbu = d.dyn[kTbu];
  a.uinit = d.dyn[kUinit];
  a.vinit = d.dyn[kVinit];
  a.u_in = d.u[from];
  a.v_in = d.v[from];
  a.u_out = d.u[to];
  a.v_out = d.v[to];
  for (int k = 0; k < 12; k++) {
    a.s_in[k] = d.stress[from][k];
    a.s_out[k] = d.stress[to][k];
  }
  a.strintx = d.strintx;
  a.strinty = d.strinty;
  a.Cb = d.Cb;
  for (int k = 0; k < 8; k++) a.str_out[k] = d.str[k];
  return a;
}

TmaArgs problem_tma_args(const DeviceProblem &d, int from) {
  TmaArgs a;
  const int to = 1 - from;
  a.ntiles = d.ntiles;
  a.nruns = d.nruns;
  a.run_off = d.run_off;
  a.tile_off = d.tile_off;
  a.tile_cnt = d.tile_cnt;
  a.halo_off = d.halo_off;
  a.halo_cnt = d.halo_cnt;
  a.halo_idx = d.halo_idx;
  a.uvx_off = d.uvx_off;
  a.uvx_cnt = d.uvx_cnt;
  a.uvx_idx = d.uvx_idx;
  a.meta = d.meta;
  a.lcor = d.lcor;
  a.halo_lcc = d.halo_lcc;
  a.halo_lcor = d.halo_lcor;
  a.tile_meta = d.tile_meta;
  a.tile_rec = d.tile_rec;
  const int geo_order[6] = {kDxT, kDyT, kHTE, kHTN, kHTEm1, kHTNm1};
  for (int k = 0; k < 6; k++) a.sg[k] = d.geo[geo_order[k]];
  a.sg[6] = d.dyn[kStrength];
  a.cblk = d.cblk;
  a.cflags = d.cflags;
  a.compact = d.compact_allowed;
  a.u[0] = d.u[from];
  a.v[0] = d.v[from];
  a.u[1] = d.u[to];
  a.v[1] = d.v[to];
  for (int k = 0; k < 12; k++) {
    a.s[0][k] = d.stress[from][k];
    a.s[1][k] = d.stress[to][k];
  }
  a.strintx = d.strintx;
  a.strinty = d.strinty;
  a.Cb = d.Cb;
  for (int k = 0; k < 8; k++) a.str_out[k] = d.str[k];
  a.dep_off = d.dep_off;
  a.dep_idx = d.dep_idx;
  a.err = d.err;
  return a;
}

int problem_take_error(DeviceProblem *d, int *code) {
  int v = 0;
  CUDA_TRY(cudaMemcpyAsync(&v, d->err, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
  CUDA_TRY(cudaStreamSynchronize(d->stream));
  if (v) CUDA_TRY(cudaMemsetAsync(d->err, 0, sizeof(int), d->stream));
  *code = v;
  return EVP1D_OK;
}

}  // namespace evp
