// evp_math.cuh -- per-point EVP arithmetic shared by every kernel variant.
//
// Each function restates one piece of the reference's Fortran with the same
// operation order (left to right within a precedence level, parentheses kept,
// x**2 as x*x, sign(1,x) as copysign).  The translation unit is compiled with
// -fmad=false, so every +, -, * is a separately rounded IEEE FP64 operation
// and / and sqrt are the IEEE correctly rounded CUDA FP64 operations: the
// results are bit-identical to the reference's -fp-model precise -no-fma
// builds.  Build flag EVP_FMA (set only in the FMA flavour of the library)
// changes nothing here; the compiler then contracts a*b+c itself.
#pragma once

#include <cmath>

#include <cuda_runtime.h>

namespace evp {

// ice_constants (src/ice.F90:25-68)
constexpr double kP111 = 1.0 / 9.0;
constexpr double kP055 = kP111 * 0.5;
constexpr double kP027 = kP055 * 0.5;
constexpr double kP166 = 1.0 / 6.0;
constexpr double kP333 = 1.0 / 3.0;
constexpr double kP222 = 2.0 / 9.0;
constexpr double kP5 = 0.5;
constexpr double kP25 = 0.25;
constexpr double kC1p5 = 1.5;
constexpr double kC1 = 1.0;

struct Params {
  double arlx1i, denom1, brlx, capping, e_factor, epp2i, deltaminEVP;
  double revp, Ktens, u0, cosw, sinw, rhow;
};

// Corner velocities of one T cell: cc = (i,j), ee = (i-1,j), ne = (i-1,j-1),
// se = (i,j-1) (integration/ice_dyn_evp1d.F90:766-769).
struct Corners {
  double ucc, vcc, uee, vee, une, vne, use, vse;
};

// Static geometry of one T cell (src/bench_v2b.F90:137-147).
struct Geom {
  double dxT, dyT, cxp, cyp, cxm, cym, DminTarea, dxhy, dyhx;
};

__host__ __device__ __forceinline__ Geom make_geom(double dxT, double dyT,
                                                   double hte, double htn,
                                                   double htem1, double htnm1,
                                                   double deltaminEVP) {
  Geom g;
  g.dxT = dxT;
  g.dyT = dyT;
  g.cxp = kC1p5 * htn - kP5 * htnm1;
  g.cyp = kC1p5 * hte - kP5 * htem1;
  g.cxm = -(kC1p5 * htnm1 - kP5 * htn);
  g.cym = -(kC1p5 * htem1 - kP5 * hte);
  // split as in the reference "for binary identity" (src/bench_v2b.F90:144)
  const double tmparea = dxT * dyT;
  g.DminTarea = deltaminEVP * tmparea;
  g.dxhy = kP5 * (hte - htem1);
  g.dyhx = kP5 * (htn - htnm1);
  return g;
}

// Fortran MAX(a,b); for a NaN operand it returns b like x86 maxsd.
__host__ __device__ __forceinline__ double fmax_ref(double a, double b) {
  return a > b ? a : b;
}

// strain_rates (src/bench_v2b.F90:321-397) and Delta.
struct Strain {
  double div[4], ten[4], shr[4], Delta[4];  // corners ne, nw, sw, se
};

__host__ __device__ __forceinline__ Strain strain_rates(const Corners &c,
                                                        const Geom &g,
                                                        double e_factor) {
  Strain s;
  const double ucc = c.ucc, vcc = c.vcc, uee = c.uee, vee = c.vee;
  const double une = c.une, vne = c.vne, use = c.use, vse = c.vse;
  const double dxT = g.dxT, dyT = g.dyT, cxp = g.cxp, cyp = g.cyp;
  const double cxm = g.cxm, cym = g.cym;
  s.div[0] = cyp * ucc - dyT * uee + cxp * vcc - dxT * vse;  // ne
  s.div[1] = cym * uee + dyT * ucc + cxp * vee - dxT * vne;  // nw
  s.div[2] = cym * une + dyT * use + cxm * vne + dxT * vee;  // sw
  s.div[3] = cyp * use - dyT * une + cxm * vse + dxT * vcc;  // se

  s.ten[0] = -(cym * ucc) - dyT * uee + cxm * vcc + dxT * vse;
  s.ten[1] = -(cyp * uee) + dyT * ucc + cxm * vee + dxT * vne;
  s.ten[2] = -(cyp * une) + dyT * use + cxp * vne - dxT * vee;
  s.ten[3] = -(cym * use) - dyT * une + cxp * vse - dxT * vcc;

  s.shr[0] = -(cym * vcc) - dyT * vee - cxm * ucc - dxT * use;
  s.shr[1] = -(cyp * vee) + dyT * vcc - cxm * uee - dxT * une;
  s.shr[2] = -(cyp * vne) + dyT * vse - cxp * une + dxT * uee;
  s.shr[3] = -(cym * vse) - dyT * vne - cxp * use + dxT * ucc;
#pragma unroll
  for (int k = 0; k < 4; k++)
    s.Delta[k] = sqrt(s.div[k] * s.div[k] +
                      e_factor * (s.ten[k] * s.ten[k] + s.shr[k] * s.shr[k]));
  return s;
}

// visc_replpress (src/bench_v2b.F90:415-437).
//
// Exact shortcuts (each result bit-identical to the literal formula):
//  - capping == 1: tmpcalc = 1*x + 0*q with x = strength/max(Delta,DminArea)
//    and q = strength/(Delta+DminArea).  1*x is x; 0*q is a zero carrying
//    q's sign, and q has x's sign, so x + 0*q is x -- provided q is finite
//    and Delta is not NaN.  Both hold when strength is finite, DminArea > 0
//    and |strength| < 1e300*DminArea (then |q| <= |strength|/DminArea), so
//    the second division is skipped under exactly those conditions.
//  - Ktens == 0: (1+Ktens)*t and (1-Ktens)*t are 1*t, which is t.
__host__ __device__ __forceinline__ void visc_replpress(
    double strength, double DminArea, double Delta, const Params &p,
    double &zetax2, double &etax2, double &rep_prs) {
  double tmpcalc;
  const bool capped = p.capping == kC1 && Delta == Delta && DminArea > 0.0 &&
                      fabs(strength) < 1e300 * DminArea;
  if (capped)
    tmpcalc = strength / fmax_ref(Delta, DminArea);
  else
    tmpcalc = p.capping * (strength / fmax_ref(Delta, DminArea)) +
              (kC1 - p.capping) * (strength / (Delta + DminArea));
  if (p.Ktens == 0.0) {
    zetax2 = tmpcalc;
    rep_prs = tmpcalc * Delta;
  } else {
    zetax2 = (kC1 + p.Ktens) * tmpcalc;
    rep_prs = (kC1 - p.Ktens) * tmpcalc * Delta;
  }
  etax2 = p.epp2i * zetax2;
}

// One corner's stress relaxation (src/bench_v2b.F90:170-212): viscosities
// from Delta, then stressp_k, stressm_k, stress12_k updated in place.
__host__ __device__ __forceinline__ void corner_update(
    double &sp, double &sm, double &s12, double div, double ten, double shr,
    double Delta, double strength, double DminTarea, const Params &p) {
  double z, e, r;
  visc_replpress(strength, DminTarea, Delta, p, z, e, r);
  const double arlx1i = p.arlx1i, denom1 = p.denom1, revp = p.revp;
  sp = (sp * (kC1 - arlx1i * revp) + arlx1i * (z * div - r)) * denom1;
  sm = (sm * (kC1 - arlx1i * revp) + arlx1i * e * ten) * denom1;
  s12 = (s12 * (kC1 - arlx1i * revp) + arlx1i * kP5 * e * shr) * denom1;
}

// Strain rates and Delta of corner k (0 ne, 1 nw, 2 sw, 3 se) in one
// branch-free form, so that the four corners of a point can run on four lanes
// of a warp.  With P1 = (cc, ee, ne, se)[k], P2 = (ee, cc, se, ne)[k] and
// P4 = (se, ne, ee, cc)[k], the reference's twelve expressions
// (src/bench_v2b.F90:363-395) are
//   div = ((A1*u[P1] + B2*u[P2]) + A3*v[P1]) + B4*v[P4]
//   ten = ((-(C1*u[P1]) + B2*u[P2]) + C3*v[P1]) + (-B4)*v[P4]
//   shr = ((-(C1*v[P1]) + B2*v[P2]) + (-C3)*u[P1]) + B4*u[P4]
// with A1 = (cyp,cym,cym,cyp), C1 = (cym,cyp,cyp,cym), A3 = (cxp,cxp,cxm,cxm),
// C3 = (cxm,cxm,cxp,cxp), B2 = (-dyT,dyT,dyT,-dyT), B4 = (-dxT,-dxT,dxT,dxT).
// Every product and sum is the reference's own: a - b is a + (-b) and
// (-a)*b is -(a*b) exactly in IEEE arithmetic.
__host__ __device__ __forceinline__ void corner_strain(
    int k, double u1, double v1, double u2, double v2, double u4, double v4,
    const Geom &g, double e_factor, double &div, double &ten, double &shr,
    double &Delta) {
  const bool a = (k == 0) | (k == 3);
  const bool b = k < 2;
  const double A1 = a ? g.cyp : g.cym;
  const double C1 = a ? g.cym : g.cyp;
  const double A3 = b ? g.cxp : g.cxm;
  const double C3 = b ? g.cxm : g.cxp;
  const double B2 = a ? -g.dyT : g.dyT;
  const double B4 = b ? -g.dxT : g.dxT;
  div = A1 * u1 + B2 * u2 + A3 * v1 + B4 * v4;
  ten = -(C1 * u1) + B2 * u2 + C3 * v1 + (-B4) * v4;
  shr = -(C1 * v1) + B2 * v2 + (-C3) * u1 + B4 * u4;
  Delta = sqrt(div * div + e_factor * (ten * ten + shr * shr));
}

// The 8 str combinations of the updated stresses (src/bench_v2b.F90:217-310).
__host__ __device__ __forceinline__ void str_combine(const double (&s)[12],
                                                     double (&out)[8],
                                                     const Geom &g);

// The 12 corner stress relaxations and the 8 str combinations
// (src/bench_v2b.F90:186-310).  s[0..11] = stressp_1..4, stressm_1..4,
// stress12_1..4 (updated in place); out[0..7] = str1..str8.
__host__ __device__ __forceinline__ void stress_update(
    double (&s)[12], double (&out)[8], const Strain &sr, double strength,
    const Geom &g, const Params &p) {
  // corner k of the reference (1=ne, 2=nw, 3=sw, 4=se) uses ne/nw/sw/se
  // strain: index map 1->0 (ne), 2->1 (nw), 3->2 (sw), 4->3 (se).
#pragma unroll
  for (int k = 0; k < 4; k++)
    corner_update(s[k], s[4 + k], s[8 + k], sr.div[k], sr.ten[k], sr.shr[k],
                  sr.Delta[k], strength, g.DminTarea, p);
  str_combine(s, out, g);
}

// True when stress_update_std may replace stress_update: capping == 1,
// Ktens == 0, revp == 0 and a finite arlx1i.
__host__ __device__ __forceinline__ bool std_params(const Params &p) {
  return p.capping == kC1 && p.Ktens == 0.0 && p.revp == 0.0 && p.arlx1i - p.arlx1i == 0.0;
}

// stress_update for parameters with std_params(p), as straight-line code: the
// four corners' divisions carry no per-corner branch, so they can overlap.
// Exactly the bits of stress_update:
//  - the capping shortcut of visc_replpress holds for all four corners when
//    DminTarea > 0, |strength| < 1e300*DminTarea and no Delta is NaN; those
//    conditions are tested once and, if any fails (never in normal runs),
//    the general stress_update runs instead on the unchanged stresses;
//  - revp == 0 with a finite arlx1i makes (1 - arlx1i*revp) exactly 1, and
//    x*1 is x for every x, so that product is dropped.
__host__ __device__ __forceinline__ void stress_update_std(
    double (&s)[12], double (&out)[8], const Strain &sr, double strength,
    const Geom &g, const Params &p) {
  const double DminArea = g.DminTarea;
  const bool ok = DminArea > 0.0 && fabs(strength) < 1e300 * DminArea &&
                  sr.Delta[0] == sr.Delta[0] && sr.Delta[1] == sr.Delta[1] &&
                  sr.Delta[2] == sr.Delta[2] && sr.Delta[3] == sr.Delta[3];
  if (!ok) {
    stress_update(s, out, sr, strength, g, p);
    return;
  }
  const double arlx1i = p.arlx1i, denom1 = p.denom1;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const double z = strength / fmax_ref(sr.Delta[k], DminArea);
    const double r = z * sr.Delta[k];
    const double e = p.epp2i * z;
    s[k] = (s[k] + arlx1i * (z * sr.div[k] - r)) * denom1;
    s[4 + k] = (s[4 + k] + arlx1i * e * sr.ten[k]) * denom1;
    s[8 + k] = (s[8 + k] + arlx1i * kP5 * e * sr.shr[k]) * denom1;
  }
  str_combine(s, out, g);
}

__host__ __device__ __forceinline__ void str_combine(const double (&s)[12],
                                                     double (&out)[8],
                                                     const Geom &g) {

  const double ssigpn = s[0] + s[1];
  const double ssigps = s[2] + s[3];
  const double ssigpe = s[0] + s[3];
  const double ssigpw = s[1] + s[2];
  const double ssigp1 = (s[0] + s[2]) * kP055;
  const double ssigp2 = (s[1] + s[3]) * kP055;

  const double ssigmn = s[4] + s[5];
  const double ssigms = s[6] + s[7];
  const double ssigme = s[4] + s[7];
  const double ssigmw = s[5] + s[6];
  const double ssigm1 = (s[4] + s[6]) * kP055;
  const double ssigm2 = (s[5] + s[7]) * kP055;

  const double ssig12n = s[8] + s[9];
  const double ssig12s = s[10] + s[11];
  const double ssig12e = s[8] + s[11];
  const double ssig12w = s[9] + s[10];
  const double ssig121 = (s[8] + s[10]) * kP111;
  const double ssig122 = (s[9] + s[11]) * kP111;

  const double csigpne = kP111 * s[0] + ssigp2 + kP027 * s[2];
  const double csigpnw = kP111 * s[1] + ssigp1 + kP027 * s[3];
  const double csigpsw = kP111 * s[2] + ssigp2 + kP027 * s[0];
  const double csigpse = kP111 * s[3] + ssigp1 + kP027 * s[1];

  const double csigmne = kP111 * s[4] + ssigm2 + kP027 * s[6];
  const double csigmnw = kP111 * s[5] + ssigm1 + kP027 * s[7];
  const double csigmsw = kP111 * s[6] + ssigm2 + kP027 * s[4];
  const double csigmse = kP111 * s[7] + ssigm1 + kP027 * s[5];

  const double csig12ne = kP222 * s[8] + ssig122 + kP055 * s[10];
  const double csig12nw = kP222 * s[9] + ssig121 + kP055 * s[11];
  const double csig12sw = kP222 * s[10] + ssig122 + kP055 * s[8];
  const double csig12se = kP222 * s[11] + ssig121 + kP055 * s[9];

  const double dxt = g.dxT, dyt = g.dyT, dxhy = g.dxhy, dyhx = g.dyhx;
  const double str12ew = kP5 * dxt * (kP333 * ssig12e + kP166 * ssig12w);
  const double str12we = kP5 * dxt * (kP333 * ssig12w + kP166 * ssig12e);
  const double str12ns = kP5 * dyt * (kP333 * ssig12n + kP166 * ssig12s);
  const double str12sn = kP5 * dyt * (kP333 * ssig12s + kP166 * ssig12n);

  double strp_tmp = kP25 * dyt * (kP333 * ssigpn + kP166 * ssigps);
  double strm_tmp = kP25 * dyt * (kP333 * ssigmn + kP166 * ssigms);
  out[0] = -strp_tmp - strm_tmp - str12ew + dxhy * (-csigpne + csigmne) +
           dyhx * csig12ne;
  out[1] = strp_tmp + strm_tmp - str12we + dxhy * (-csigpnw + csigmnw) +
           dyhx * csig12nw;

  strp_tmp = kP25 * dyt * (kP333 * ssigps + kP166 * ssigpn);
  strm_tmp = kP25 * dyt * (kP333 * ssigms + kP166 * ssigmn);
  out[2] = -strp_tmp - strm_tmp + str12ew + dxhy * (-csigpse + csigmse) +
           dyhx * csig12se;
  out[3] = strp_tmp + strm_tmp + str12we + dxhy * (-csigpsw + csigmsw) +
           dyhx * csig12sw;

  strp_tmp = kP25 * dxt * (kP333 * ssigpe + kP166 * ssigpw);
  strm_tmp = kP25 * dxt * (kP333 * ssigme + kP166 * ssigmw);
  out[4] = -strp_tmp + strm_tmp - str12ns - dyhx * (csigpne + csigmne) +
           dxhy * csig12ne;
  out[5] = strp_tmp - strm_tmp - str12sn - dyhx * (csigpse + csigmse) +
           dxhy * csig12se;

  strp_tmp = kP25 * dxt * (kP333 * ssigpw + kP166 * ssigpe);
  strm_tmp = kP25 * dxt * (kP333 * ssigmw + kP166 * ssigme);
  out[6] = -strp_tmp + strm_tmp + str12ns - dyhx * (csigpnw + csigmnw) +
           dxhy * csig12nw;
  out[7] = strp_tmp - strm_tmp + str12sn - dyhx * (csigpsw + csigmsw) +
           dxhy * csig12sw;
}

// Inputs of stepu at one U point (src/bench_v2b.F90:506-544).  kvrel is the
// per-point factor aiX*rhow*Cw of the drag term, evaluated left to right
// ((aiX*rhow)*Cw) as the reference does (:513); it does not change within a
// call, so the fused path computes it once per call.
__host__ __device__ __forceinline__ double drag_factor(double aiX, double rhow,
                                                       double Cw) {
  return aiX * rhow * Cw;
}

struct StepuIn {
  double uold, vold;
  double kvrel, uocn, vocn, waterx, watery, forcex, forcey;
  double umassdti, fm, uarear, Tbu, uinit, vinit;
  // str1(iw), str2(nw), str3(sse), str4(sw), str5(iw), str6(sse), str7(nw),
  // str8(sw)
  double s1, s2nw, s3sse, s4sw, s5, s6sse, s7nw, s8sw;
};

struct StepuOut {
  double u, v, strintx, strinty, Cb;
};

// stepu at one point (src/bench_v2b.F90:509-544).
//
// Exact shortcuts (each result bit-identical to the literal formula):
//  - Tbu == +0, u0 > 0 and u, v not NaN: the denominator sqrt(u^2+v^2)+u0
//    is positive or +Inf, so Cb = +0 without the square root and division;
//  - cosw == 1: vrel*cosw is vrel;
//  - sinw == 0: sign(1,fm)*vrel*0 is a signed zero, and fm + (that zero) is
//    fm unless fm is -0 and the zero is +0, i.e. unless fm == -0 and
//    vrel < 0; a NaN vrel takes the literal route; an infinite vrel makes u
//    and v NaN on both routes, and strintx, strinty and Cb do not use ccb.
__host__ __device__ __forceinline__ StepuOut stepu_point(const StepuIn &in,
                                                         const Params &p) {
  StepuOut o;
  const double uold = in.uold, vold = in.vold;
  const double du = in.uocn - uold, dv = in.vocn - vold;
  const double vrel = in.kvrel * sqrt(du * du + dv * dv);
  const double taux = vrel * in.waterx;
  const double tauy = vrel * in.watery;
  const bool tbu_zero = in.Tbu == 0.0 && copysign(kC1, in.Tbu) > 0.0 && p.u0 > 0.0 &&
                        uold == uold && vold == vold;
  o.Cb = tbu_zero ? 0.0 : in.Tbu / (sqrt(uold * uold + vold * vold) + p.u0);
  const double cca = (p.brlx + p.revp) * in.umassdti + (p.cosw == kC1 ? vrel : vrel * p.cosw) + o.Cb;
  const double ccb = p.sinw == 0.0 && (in.fm != 0.0 || vrel >= 0.0)
                         ? in.fm
                         : in.fm + copysign(kC1, in.fm) * vrel * p.sinw;
  const double ab2 = cca * cca + ccb * ccb;
  o.strintx = in.uarear * (in.s1 + in.s2nw + in.s3sse + in.s4sw);
  o.strinty = in.uarear * (in.s5 + in.s6sse + in.s7nw + in.s8sw);
  const double cc1 = o.strintx + in.forcex + taux +
                     in.umassdti * (p.brlx * uold + p.revp * in.uinit);
  const double cc2 = o.strinty + in.forcey + tauy +
                     in.umassdti * (p.brlx * vold + p.revp * in.vinit);
  o.u = (cca * cc1 + ccb * cc2) / ab2;
  o.v = (cca * cc2 - ccb * cc1) / ab2;
  return o;
}

}  // namespace evp
