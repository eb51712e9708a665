// evp_adjoint_math.cuh -- reverse-mode derivatives of one EVP subcycle at a
// point (hand-written, FP64).
//
// The forward quantities a derivative needs are recomputed from the stored
// velocities in the forward's own operation order (evp_math.cuh; the
// branch-deciding ones below with the forward's rounding), so every branch
// takes the side the forward took: max(Delta, DminArea) (src/bench_v2b.F90:
// 428-430), the capped/uncapped viscosity, and a zero-length square root
// (Delta = 0, |u| = 0, |u_ocn - u| = 0), whose derivative is taken as 0.
//
// A "lam" value is the adjoint dJ/d(value) of a scalar loss J.  The stress
// relaxation is linear in the old stresses with state-independent
// coefficients, so the reverse sweep needs the velocities of each subcycle
// but never the stresses.  These derivatives are not bit-matched to anything:
// a reciprocal is multiplied where the forward divides, and the reverse
// kernels are compiled with a*b+c contracted to fused multiply-adds.
//
// The forward values that choose a branch -- Delta against DminTarea and 0,
// |u| and |u_ocn - u| against 0 -- are recomputed with every +, -, * rounded
// on its own (fw_mul/fw_add/fw_sub: the __d*_rn intrinsics, which the
// compiler never contracts), in the forward's operation order, so they equal
// the bit-exact forward's values whatever the file's contraction setting.
// In the FMA flavour of the library (EVP_FMA) the forward itself is
// contracted, so these are plain operations there as well.
#pragma once

#include "evp_math.cuh"

namespace evp {

__host__ __device__ __forceinline__ double fw_mul(double a, double b) {
#if defined(__CUDA_ARCH__) && !defined(EVP_FMA)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
__host__ __device__ __forceinline__ double fw_add(double a, double b) {
#if defined(__CUDA_ARCH__) && !defined(EVP_FMA)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
__host__ __device__ __forceinline__ double fw_sub(double a, double b) {
#if defined(__CUDA_ARCH__) && !defined(EVP_FMA)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}

// make_geom (src/bench_v2b.F90:137-147) with every operation rounded on its
// own: the same bits as the forward's geometry.
__host__ __device__ __forceinline__ Geom make_geom_fw(double dxT, double dyT, double hte,
                                                      double htn, double htem1, double htnm1,
                                                      double deltaminEVP) {
  Geom g;
  g.dxT = dxT;
  g.dyT = dyT;
  g.cxp = fw_sub(fw_mul(kC1p5, htn), fw_mul(kP5, htnm1));
  g.cyp = fw_sub(fw_mul(kC1p5, hte), fw_mul(kP5, htem1));
  g.cxm = -fw_sub(fw_mul(kC1p5, htnm1), fw_mul(kP5, htn));
  g.cym = -fw_sub(fw_mul(kC1p5, htem1), fw_mul(kP5, hte));
  g.DminTarea = fw_mul(deltaminEVP, fw_mul(dxT, dyT));
  g.dxhy = fw_mul(kP5, fw_sub(hte, htem1));
  g.dyhx = fw_mul(kP5, fw_sub(htn, htnm1));
  return g;
}

// corner_strain (the strain rates and Delta of one corner, src/bench_v2b.F90:
// 363-397) with every operation rounded on its own, left to right as in the
// forward: the same div, ten, shr and Delta bits.
__host__ __device__ __forceinline__ void corner_strain_fw(
    int k, double u1, double v1, double u2, double v2, double u4, double v4, const Geom &g,
    double e_factor, double &div, double &ten, double &shr, double &Delta) {
  const bool a = (k == 0) | (k == 3);
  const bool b = k < 2;
  const double A1 = a ? g.cyp : g.cym;
  const double C1 = a ? g.cym : g.cyp;
  const double A3 = b ? g.cxp : g.cxm;
  const double C3 = b ? g.cxm : g.cxp;
  const double B2 = a ? -g.dyT : g.dyT;
  const double B4 = b ? -g.dxT : g.dxT;
  div = fw_add(fw_add(fw_add(fw_mul(A1, u1), fw_mul(B2, u2)), fw_mul(A3, v1)), fw_mul(B4, v4));
  ten = fw_add(fw_add(fw_add(-fw_mul(C1, u1), fw_mul(B2, u2)), fw_mul(C3, v1)),
               fw_mul(-B4, v4));
  shr = fw_add(fw_add(fw_add(-fw_mul(C1, v1), fw_mul(B2, v2)), fw_mul(-C3, u1)),
               fw_mul(B4, u4));
  Delta = sqrt(fw_add(fw_mul(div, div),
                      fw_mul(e_factor, fw_add(fw_mul(ten, ten), fw_mul(shr, shr)))));
}

// Transpose of str_combine (src/bench_v2b.F90:217-310): given lo[0..7] =
// dJ/d str1..str8 at a point, add dJ/d s[0..11] (the updated stresses) to ls.
__host__ __device__ __forceinline__ void str_combine_adjoint(const double (&lo)[8],
                                                             const Geom &g,
                                                             double (&ls)[12]) {
  const double dxt = g.dxT, dyt = g.dyT, dxhy = g.dxhy, dyhx = g.dyhx;
  // strp_tmp / strm_tmp of the four str pairs, and str12ew/we/ns/sn
  const double l_pa = -lo[0] + lo[1], l_ma = -lo[0] + lo[1];
  const double l_pb = -lo[2] + lo[3], l_mb = -lo[2] + lo[3];
  const double l_pc = -lo[4] + lo[5], l_mc = lo[4] - lo[5];
  const double l_pd = -lo[6] + lo[7], l_md = lo[6] - lo[7];
  const double l_12ew = -lo[0] + lo[2], l_12we = -lo[1] + lo[3];
  const double l_12ns = -lo[4] + lo[6], l_12sn = -lo[5] + lo[7];
  // csig{p,m,12}{ne,nw,se,sw}
  const double l_cpne = -dxhy * lo[0] - dyhx * lo[4], l_cmne = dxhy * lo[0] - dyhx * lo[4];
  const double l_c12ne = dyhx * lo[0] + dxhy * lo[4];
  const double l_cpnw = -dxhy * lo[1] - dyhx * lo[6], l_cmnw = dxhy * lo[1] - dyhx * lo[6];
  const double l_c12nw = dyhx * lo[1] + dxhy * lo[6];
  const double l_cpse = -dxhy * lo[2] - dyhx * lo[5], l_cmse = dxhy * lo[2] - dyhx * lo[5];
  const double l_c12se = dyhx * lo[2] + dxhy * lo[5];
  const double l_cpsw = -dxhy * lo[3] - dyhx * lo[7], l_cmsw = dxhy * lo[3] - dyhx * lo[7];
  const double l_c12sw = dyhx * lo[3] + dxhy * lo[7];
  const double ky3 = kP25 * dyt * kP333, ky6 = kP25 * dyt * kP166;
  const double kx3 = kP25 * dxt * kP333, kx6 = kP25 * dxt * kP166;
  const double hx3 = kP5 * dxt * kP333, hx6 = kP5 * dxt * kP166;
  const double hy3 = kP5 * dyt * kP333, hy6 = kP5 * dyt * kP166;
  // ssig{p,m,12}{n,s,e,w}
  const double l_pn = ky3 * l_pa + ky6 * l_pb, l_ps = ky6 * l_pa + ky3 * l_pb;
  const double l_pe = kx3 * l_pc + kx6 * l_pd, l_pw = kx6 * l_pc + kx3 * l_pd;
  const double l_mn = ky3 * l_ma + ky6 * l_mb, l_ms = ky6 * l_ma + ky3 * l_mb;
  const double l_me = kx3 * l_mc + kx6 * l_md, l_mw = kx6 * l_mc + kx3 * l_md;
  const double l_12e = hx3 * l_12ew + hx6 * l_12we, l_12w = hx6 * l_12ew + hx3 * l_12we;
  const double l_12n = hy3 * l_12ns + hy6 * l_12sn, l_12s = hy6 * l_12ns + hy3 * l_12sn;
  // ssig{p,m,12}{1,2}
  const double l_p1 = l_cpnw + l_cpse, l_p2 = l_cpne + l_cpsw;
  const double l_m1 = l_cmnw + l_cmse, l_m2 = l_cmne + l_cmsw;
  const double l_121 = l_c12nw + l_c12se, l_122 = l_c12ne + l_c12sw;
  ls[0] += l_pn + l_pe + kP055 * l_p1 + kP111 * l_cpne + kP027 * l_cpsw;
  ls[1] += l_pn + l_pw + kP055 * l_p2 + kP111 * l_cpnw + kP027 * l_cpse;
  ls[2] += l_ps + l_pw + kP055 * l_p1 + kP111 * l_cpsw + kP027 * l_cpne;
  ls[3] += l_ps + l_pe + kP055 * l_p2 + kP111 * l_cpse + kP027 * l_cpnw;
  ls[4] += l_mn + l_me + kP055 * l_m1 + kP111 * l_cmne + kP027 * l_cmsw;
  ls[5] += l_mn + l_mw + kP055 * l_m2 + kP111 * l_cmnw + kP027 * l_cmse;
  ls[6] += l_ms + l_mw + kP055 * l_m1 + kP111 * l_cmsw + kP027 * l_cmne;
  ls[7] += l_ms + l_me + kP055 * l_m2 + kP111 * l_cmse + kP027 * l_cmnw;
  ls[8] += l_12n + l_12e + kP111 * l_121 + kP222 * l_c12ne + kP055 * l_c12sw;
  ls[9] += l_12n + l_12w + kP111 * l_122 + kP222 * l_c12nw + kP055 * l_c12se;
  ls[10] += l_12s + l_12w + kP111 * l_121 + kP222 * l_c12sw + kP055 * l_c12ne;
  ls[11] += l_12s + l_12e + kP111 * l_122 + kP222 * l_c12se + kP055 * l_c12nw;
}

// Reverse of one corner's relaxation (corner_update with visc_replpress,
// src/bench_v2b.F90:186-212, 415-437).  In: l_sp, l_sm, l_s12 = lam of the
// updated stresses of the corner.  Out: lam of the old stresses (returned in
// place), lam of the corner's div, ten, shr (through Delta as well) and the
// corner's contribution to dJ/dstrength.
__host__ __device__ __forceinline__ void corner_adjoint(
    double &l_sp, double &l_sm, double &l_s12, double div, double ten, double shr,
    double Delta, double strength, double DminArea, const Params &p, double &l_div,
    double &l_ten, double &l_shr, double &l_strength) {
  const double a = p.arlx1i, d = p.denom1;
  const double keep = (kC1 - a * p.revp) * d;
  const double A = l_sp * d * a;          // lam of (zetax2*div - rep_prs)
  const double B = l_sm * d * a;          // lam of etax2*ten
  const double Cc = l_s12 * d * a * kP5;  // lam of etax2*shr
  l_sp *= keep;
  l_sm *= keep;
  l_s12 *= keep;
  // the forward's viscosity (tmpcalc) and its derivatives
  const bool above = Delta > DminArea;  // max(Delta, DminArea) picked Delta
  const double inv_m = kC1 / (above ? Delta : DminArea);
  double tmp, dtmp_dstr, dtmp_dD;
  if (p.capping == kC1) {
    tmp = strength * inv_m;
    dtmp_dstr = inv_m;
    dtmp_dD = above ? -tmp * inv_m : 0.0;
  } else {
    const double inv_p = kC1 / (Delta + DminArea);
    tmp = p.capping * (strength * inv_m) + (kC1 - p.capping) * (strength * inv_p);
    dtmp_dstr = p.capping * inv_m + (kC1 - p.capping) * inv_p;
    dtmp_dD = (above ? -p.capping * strength * inv_m * inv_m : 0.0) -
              (kC1 - p.capping) * strength * inv_p * inv_p;
  }
  const double z = (kC1 + p.Ktens) * tmp, e = p.epp2i * z;
  // zetax2 = (1+Ktens)*tmp, etax2 = epp2i*zetax2, rep_prs = (1-Ktens)*tmp*Delta
  const double l_e = B * ten + Cc * shr;
  const double l_z = A * div + p.epp2i * l_e;
  const double l_r = -A;
  const double l_tmp = (kC1 + p.Ktens) * l_z + (kC1 - p.Ktens) * Delta * l_r;
  const double l_Delta = (kC1 - p.Ktens) * tmp * l_r + l_tmp * dtmp_dD;
  l_strength = l_tmp * dtmp_dstr;
  l_div = A * z;
  l_ten = B * e;
  l_shr = Cc * e;
  // Delta = sqrt(div^2 + e_factor*(ten^2 + shr^2))
  if (Delta > 0.0) {
    const double q = l_Delta * (above ? inv_m : kC1 / Delta);
    l_div += q * div;
    l_ten += q * p.e_factor * ten;
    l_shr += q * p.e_factor * shr;
  }
}

// Reverse of stress at one T point.  lo = lam of str1..str8 written by the
// subcycle, ls = lam of the updated stresses (in: from later subcycles; out:
// lam of the old stresses).  Returns the lam of the 8 corner velocities and
// the point's dJ/dstrength contribution.
//
// Corner by corner: corner_strain_fw gives the corner's div, ten, shr and
// Delta (bit for bit those of strain_rates, so every branch follows the
// forward; g must come from make_geom_fw),
// corner_adjoint reverses its relaxation, and the corner's share of the
// transposed strain rates is added to lc at once.  Only one corner's strain
// is live at a time.  With P1 = (cc, ee, ne, se)[k], P2 = (ee, cc, se, ne)[k],
// P4 = (se, ne, ee, cc)[k] and the coefficients of corner_strain:
//   lam u[P1] += A1 D - C1 T - C3 H,  lam v[P1] += A3 D + C3 T - C1 H,
//   lam u[P2] += B2 (D + T),          lam v[P2] += B2 H,
//   lam u[P4] += B4 H,                lam v[P4] += B4 (D - T).
__host__ __device__ __forceinline__ void stress_adjoint(const Corners &c, const Geom &g,
                                                        double strength, const Params &p,
                                                        const double (&lo)[8],
                                                        double (&ls)[12], double (&lc)[8],
                                                        double &l_strength) {
  str_combine_adjoint(lo, g, ls);
  const double uu[4] = {c.ucc, c.uee, c.une, c.use};
  const double vv[4] = {c.vcc, c.vee, c.vne, c.vse};
#pragma unroll
  for (int q = 0; q < 8; q++) lc[q] = 0.0;
  l_strength = 0.0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int p1 = k, p2 = k ^ 1, p4 = 3 - k;
    double div, ten, shr, Delta;
    corner_strain_fw(k, uu[p1], vv[p1], uu[p2], vv[p2], uu[p4], vv[p4], g, p.e_factor, div,
                     ten, shr, Delta);
    double D, T, H, lst;
    corner_adjoint(ls[k], ls[4 + k], ls[8 + k], div, ten, shr, Delta, strength, g.DminTarea, p,
                   D, T, H, lst);
    l_strength += lst;
    const bool a = (k == 0) | (k == 3);
    const bool b = k < 2;
    const double A1 = a ? g.cyp : g.cym;
    const double C1 = a ? g.cym : g.cyp;
    const double A3 = b ? g.cxp : g.cxm;
    const double C3 = b ? g.cxm : g.cxp;
    const double B2 = a ? -g.dyT : g.dyT;
    const double B4 = b ? -g.dxT : g.dxT;
    lc[2 * p1] += A1 * D - C1 * T - C3 * H;
    lc[2 * p1 + 1] += A3 * D + C3 * T - C1 * H;
    lc[2 * p2] += B2 * (D + T);
    lc[2 * p2 + 1] += B2 * H;
    lc[2 * p4] += B4 * H;
    lc[2 * p4 + 1] += B4 * (D - T);
  }
}

// Reverse of stepu at one U point (src/bench_v2b.F90:509-544) from the
// velocity before (uold, vold) and after (unew, vnew) the subcycle.  cc1 and
// cc2 are recovered from the solved velocity, [cc1; cc2] = [[cca, -ccb],
// [ccb, cca]] [unew; vnew].
struct StepuAdjIn {
  double uold, vold, unew, vnew;
  double lun, lvn;  // lam of unew, vnew
  double kvrel, aiXrhow, uocn, vocn, waterx, watery, umassdti, fm, Tbu;
};
struct StepuAdjOut {
  double luold, lvold;  // lam of uold, vold through this stepu
  double lcc1, lcc2;    // lam of strintx + forcex + ..., i.e. of strintx, forcex
  double gCw;           // dJ/dCw contribution
  double luinit, lvinit;
};

__host__ __device__ __forceinline__ StepuAdjOut stepu_adjoint(const StepuAdjIn &in,
                                                              const Params &p) {
  StepuAdjOut o;
  const double u = in.uold, v = in.vold;
  // |u_ocn - u| and |u| as the forward rounds them (they are tested against 0)
  const double du = fw_sub(in.uocn, u), dv = fw_sub(in.vocn, v);
  const double sq = sqrt(fw_add(fw_mul(du, du), fw_mul(dv, dv)));
  const double vrel = in.kvrel * sq;
  const double sn = sqrt(fw_add(fw_mul(u, u), fw_mul(v, v)));
  const double den = sn + p.u0;
  const double Cb = in.Tbu / den;
  const double cca = (p.brlx + p.revp) * in.umassdti + vrel * p.cosw + Cb;
  const double sg = copysign(kC1, in.fm);
  const double ccb = in.fm + sg * vrel * p.sinw;
  const double inv_ab2 = kC1 / (cca * cca + ccb * ccb);
  const double cc1 = cca * in.unew - ccb * in.vnew;
  const double cc2 = ccb * in.unew + cca * in.vnew;
  // unew = (cca*cc1 + ccb*cc2)/ab2, vnew = (cca*cc2 - ccb*cc1)/ab2
  const double lN1 = in.lun * inv_ab2, lN2 = in.lvn * inv_ab2;
  const double lab2 = -(in.lun * in.unew + in.lvn * in.vnew) * inv_ab2;
  const double lcca = lN1 * cc1 + lN2 * cc2 + lab2 * 2.0 * cca;
  const double lccb = lN1 * cc2 - lN2 * cc1 + lab2 * 2.0 * ccb;
  o.lcc1 = lN1 * cca - lN2 * ccb;
  o.lcc2 = lN1 * ccb + lN2 * cca;
  // cc1 = strintx + forcex + vrel*waterx + umassdti*(brlx*u + revp*uinit)
  double lu = o.lcc1 * in.umassdti * p.brlx, lv = o.lcc2 * in.umassdti * p.brlx;
  o.luinit = o.lcc1 * in.umassdti * p.revp;
  o.lvinit = o.lcc2 * in.umassdti * p.revp;
  const double lvrel = o.lcc1 * in.waterx + o.lcc2 * in.watery + lcca * p.cosw +
                       lccb * sg * p.sinw;
  // Cb = Tbu/(sqrt(u^2+v^2) + u0)
  if (in.Tbu != 0.0 && sn > 0.0) {
    const double lsn = -lcca * Cb / (den * sn);
    lu += lsn * u;
    lv += lsn * v;
  }
  // vrel = (aiX*rhow*Cw) * sqrt(du^2 + dv^2)
  o.gCw = lvrel * sq * in.aiXrhow;
  if (sq > 0.0) {
    const double lsq = lvrel * in.kvrel / sq;
    lu -= lsq * du;
    lv -= lsq * dv;
  }
  o.luold = lu;
  o.lvold = lv;
  return o;
}

}  // namespace evp
