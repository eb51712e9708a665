// evp_dyn.cpp -- the 2D adapter of include/evp1d.h (evp1d_dyn_*): the
// dyn_evp1d_init / dyn_evp1d_run / dyn_evp1d_finalize interface on global 2D
// arrays, on top of the 1D C-ABI.  The 2D <-> 1D copies are O(nActive) host
// loops over the list points (convert_2d_1d_dyn / convert_1d_2d_dyn,
// integration/ice_dyn_evp1d.F90:818-947).
#include <cstdint>
#include <string>
#include <vector>

#include "evp1d.h"

namespace evp {
int error(int code, const char *fmt, ...);  // evp1d_api.cu
}

struct evp1d_dyn_handle {
  int nx = 0, ny = 0, na = 0, navel = 0;
  std::vector<int32_t> ti, tj;  // 1-based (i, j) of each list point
  evp1d_t *h = nullptr;
  // 1D scratch of one call
  std::vector<int32_t> skipT, skipU;
  std::vector<double> buf;
};

namespace {

inline size_t at(const evp1d_dyn_handle *d, int w) {
  return (size_t)(d->ti[w] - 1) + (size_t)(d->tj[w] - 1) * (size_t)d->nx;
}

}  // namespace

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
  int na = 0, navel = 0;
  int rc = evp1d_build_index(nx, ny, nghost, tmask, 0, 0, &na, &navel, nullptr, nullptr,
                             nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (rc != EVP1D_OK && rc != EVP1D_ERR_INVALID_ARG) return rc;
  evp1d_dyn_t *d = new evp1d_dyn_handle();
  d->nx = nx;
  d->ny = ny;
  d->na = na;
  d->navel = navel;
  d->ti.resize((size_t)na + 1);
  d->tj.resize((size_t)na + 1);
  std::vector<int32_t> tij((size_t)navel + 1), nb((size_t)6 * (na + 1));
  int32_t *nbp[6];
  for (int k = 0; k < 6; k++) nbp[k] = nb.data() + (size_t)k * (na + 1);
  rc = evp1d_build_index(nx, ny, nghost, tmask, na, navel, &na, &navel, d->ti.data(),
                         d->tj.data(), tij.data(), nbp[0], nbp[1], nbp[2], nbp[3], nbp[4],
                         nbp[5]);
  if (rc != EVP1D_OK) {
    delete d;
    return rc;
  }
  // static 1D geometry (convert_2d_1d_init, :803-815): HTEm1 = HTE(i-1,j),
  // HTNm1 = HTN(i,j-1)
  std::vector<double> g((size_t)7 * (na + 1));
  double *G[7];
  for (int k = 0; k < 7; k++) G[k] = g.data() + (size_t)k * (na + 1);
  for (int w = 0; w < na; w++) {
    const size_t c = at(d, w);
    G[0][w] = dxT[c];
    G[1][w] = dyT[c];
    G[2][w] = HTE[c];
    G[3][w] = HTN[c];
    G[4][w] = HTE[c - 1];
    G[5][w] = HTN[c - (size_t)nx];
    G[6][w] = uarear[c];
  }
  rc = evp1d_init(&d->h, na, navel, nbp[0], nbp[1], nbp[2], nbp[3], nbp[4], nbp[5], G[0],
                  G[1], G[2], G[3], G[4], G[5], G[6], params, device);
  if (rc != EVP1D_OK) {
    delete d;
    return rc;
  }
  *handle = d;
  return EVP1D_OK;
}

int evp1d_dyn_run(evp1d_dyn_t *d, int ndte, const evp1d_dyn_fields *io) {
  if (!d || !io) return evp::error(EVP1D_ERR_INVALID_ARG, "NULL argument");
  const double *in[12] = {io->strength, io->cdn_ocn, io->aiu, io->uocn, io->vocn,
                          io->waterxU, io->wateryU, io->forcexU, io->forceyU,
                          io->umassdti, io->fmU, io->Tbu};
  for (int k = 0; k < 12; k++)
    if (!in[k] || !io->stress[k]) return evp::error(EVP1D_ERR_INVALID_ARG, "NULL field");
  if (!io->strintxU || !io->strintyU || !io->Cb || !io->uvel || !io->vvel ||
      !io->icetmask || !io->iceumask)
    return evp::error(EVP1D_ERR_INVALID_ARG, "NULL field");
  const int na = d->na, navel = d->navel;
  if (na == 0) return EVP1D_OK;
  // 1D scratch: 12 inputs, 12 stresses, strintx, strinty, Cb, u[navel], v[navel]
  d->buf.assign((size_t)27 * na + 2 * (size_t)navel, 0.0);
  double *p = d->buf.data();
  double *I[12], *S[12];
  for (int k = 0; k < 12; k++) I[k] = p + (size_t)k * na;
  for (int k = 0; k < 12; k++) S[k] = p + (size_t)(12 + k) * na;
  double *sx = p + (size_t)24 * na, *sy = p + (size_t)25 * na, *cb = p + (size_t)26 * na;
  double *u = p + (size_t)27 * na, *v = u + navel;  // halo slots stay 0 (:880-881)
  d->skipT.resize((size_t)na);
  d->skipU.resize((size_t)na);
  for (int w = 0; w < na; w++) {
    const size_t c = at(d, w);
    d->skipT[w] = io->icetmask[c] ? 0 : 1;  // set_skipMe (:521-537)
    d->skipU[w] = io->iceumask[c] ? 0 : 1;
    for (int k = 0; k < 12; k++) I[k][w] = in[k][c];
    for (int k = 0; k < 12; k++) S[k][w] = io->stress[k][c];
    sx[w] = io->strintxU[c];
    sy[w] = io->strintyU[c];
    cb[w] = io->Cb[c];
    u[w] = io->uvel[c];
    v[w] = io->vvel[c];
  }
  evp1d_fields f = {};
  f.skipT = d->skipT.data();
  f.skipU = d->skipU.data();
  for (int k = 0; k < 12; k++) f.stress[k] = S[k];
  f.strength = I[0];
  f.Cw = I[1];
  f.aiu = I[2];
  f.uocn = I[3];
  f.vocn = I[4];
  f.waterx = I[5];
  f.watery = I[6];
  f.forcex = I[7];
  f.forcey = I[8];
  f.umassdti = I[9];
  f.fm = I[10];
  f.Tbu = I[11];
  f.uvel = u;
  f.vvel = v;
  f.strintx = sx;
  f.strinty = sy;
  f.Cb = cb;
  const int rc = evp1d_run(d->h, ndte, &f);
  if (rc != EVP1D_OK) return rc;
  for (int w = 0; w < na; w++) {  // convert_1d_2d_dyn (:884-947), results only
    const size_t c = at(d, w);
    for (int k = 0; k < 12; k++) io->stress[k][c] = S[k][w];
    io->strintxU[c] = sx[w];
    io->strintyU[c] = sy[w];
    io->Cb[c] = cb[w];
    io->uvel[c] = u[w];
    io->vvel[c] = v[w];
  }
  return EVP1D_OK;
}

int evp1d_dyn_finalize(evp1d_dyn_t *d) {
  if (!d) return EVP1D_OK;
  const int rc = evp1d_finalize(d->h);
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
