// Host build of the library's per-point adjoint arithmetic
// (cice-evp1d_b200/csrc/evp_adjoint_math.cuh) for CPU unit tests against
// torch autograd.  Test code only.
#include <cuda_runtime.h>

#include "evp_adjoint_math.cuh"

namespace {
evp::Params params_of(const double *q) {
  evp::Params p;
  p.arlx1i = q[0];
  p.denom1 = q[1];
  p.brlx = q[2];
  p.capping = q[3];
  p.e_factor = q[4];
  p.epp2i = q[5];
  p.deltaminEVP = q[6];
  p.revp = q[7];
  p.Ktens = q[8];
  p.u0 = q[9];
  p.cosw = q[10];
  p.sinw = q[11];
  p.rhow = q[12];
  return p;
}
}  // namespace

extern "C" {

// n points; corners [8][n] (ucc vcc uee vee une vne use vse); geo [6][n]
// (dxT dyT HTE HTN HTEm1 HTNm1); lo [8][n]; ls [12][n] in/out; lc [8][n]
// out; lstr [n] out.
void shim_stress_adjoint(int n, const double *corners, const double *geo,
                         const double *strength, const double *q, const double *lo_in,
                         double *ls_io, double *lc_out, double *lstr) {
  const evp::Params p = params_of(q);
  for (int w = 0; w < n; w++) {
    evp::Corners c;
    c.ucc = corners[0 * n + w];
    c.vcc = corners[1 * n + w];
    c.uee = corners[2 * n + w];
    c.vee = corners[3 * n + w];
    c.une = corners[4 * n + w];
    c.vne = corners[5 * n + w];
    c.use = corners[6 * n + w];
    c.vse = corners[7 * n + w];
    const evp::Geom g = evp::make_geom_fw(geo[0 * n + w], geo[1 * n + w], geo[2 * n + w],
                                       geo[3 * n + w], geo[4 * n + w], geo[5 * n + w],
                                       p.deltaminEVP);
    double lo[8], ls[12], lc[8], l;
    for (int k = 0; k < 8; k++) lo[k] = lo_in[k * n + w];
    for (int k = 0; k < 12; k++) ls[k] = ls_io[k * n + w];
    evp::stress_adjoint(c, g, strength[w], p, lo, ls, lc, l);
    for (int k = 0; k < 12; k++) ls_io[k * n + w] = ls[k];
    for (int k = 0; k < 8; k++) lc_out[k * n + w] = lc[k];
    lstr[w] = l;
  }
}

// in [15][n]: uold vold unew vnew lun lvn kvrel aiXrhow uocn vocn waterx
// watery umassdti fm Tbu; out [7][n]: luold lvold lcc1 lcc2 gCw luinit lvinit
void shim_stepu_adjoint(int n, const double *in, const double *q, double *out) {
  const evp::Params p = params_of(q);
  for (int w = 0; w < n; w++) {
    evp::StepuAdjIn a;
    double *f[15] = {&a.uold, &a.vold, &a.unew, &a.vnew, &a.lun, &a.lvn, &a.kvrel,
                     &a.aiXrhow, &a.uocn, &a.vocn, &a.waterx, &a.watery, &a.umassdti,
                     &a.fm, &a.Tbu};
    for (int k = 0; k < 15; k++) *f[k] = in[k * n + w];
    const evp::StepuAdjOut o = evp::stepu_adjoint(a, p);
    const double r[7] = {o.luold, o.lvold, o.lcc1, o.lcc2, o.gCw, o.luinit, o.lvinit};
    for (int k = 0; k < 7; k++) out[k * n + w] = r[k];
  }
}

}  // extern "C"
