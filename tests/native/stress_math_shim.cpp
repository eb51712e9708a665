// Host build of the library's per-point stress arithmetic
// (cice-evp1d_b200/csrc/evp_math.cuh) for CPU unit tests: the general
// stress_update and the straight-line stress_update_std side by side.  Test
// code only.
#include <cuda_runtime.h>

#include "evp_math.cuh"

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

int shim_std_params(const double *q) { return evp::std_params(params_of(q)) ? 1 : 0; }

// n points; corners [8][n] (ucc vcc uee vee une vne use vse); geo [6][n]
// (dxT dyT HTE HTN HTEm1 HTNm1); s [12][n] stresses in; std != 0 selects
// stress_update_std.  Writes the updated stresses to s_out [12][n] and
// str1..8 to str_out [8][n].
void shim_stress(int n, int std, const double *corners, const double *geo,
                 const double *strength, const double *q, const double *s_in,
                 double *s_out, double *str_out) {
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
    const evp::Geom g = evp::make_geom(geo[0 * n + w], geo[1 * n + w], geo[2 * n + w],
                                       geo[3 * n + w], geo[4 * n + w], geo[5 * n + w],
                                       p.deltaminEVP);
    const evp::Strain sr = evp::strain_rates(c, g, p.e_factor);
    double s[12], out[8];
    for (int k = 0; k < 12; k++) s[k] = s_in[k * n + w];
    if (std)
      evp::stress_update_std(s, out, sr, strength[w], g, p);
    else
      evp::stress_update(s, out, sr, strength[w], g, p);
    for (int k = 0; k < 12; k++) s_out[k * n + w] = s[k];
    for (int k = 0; k < 8; k++) str_out[k * n + w] = out[k];
  }
}

}  // extern "C"
