/*
 * EVP-1D ORACLE -- test infrastructure only (see evp_oracle.h).
 *
 * CPU restatement of the reference's arithmetic in the Fortran operation
 * order.  Compile with -ffp-contract=off -fno-fast-math (no FMA contraction),
 * which is the C equivalent of the reference's f0/f1 flag sets
 * (compiler_oneapi.mk:17-18: -fp-model precise -no-fma).
 *
 * Citations are file:line inside dmidk/cice-evp1d.
 */
#include "evp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ice_constants (src/ice.F90:25-68): p111=c1/c9, p055=p111*p5,
 * p027=p055*p5, p166=c1/c6, p333=c1/c3, p222=c2/c9. */
static const double c1 = 1.0, p5 = 0.5, p25 = 0.25, c1p5 = 1.5;
#define P111 (1.0 / 9.0)
#define P055 (P111 * 0.5)
#define P027 (P055 * 0.5)
#define P166 (1.0 / 6.0)
#define P333 (1.0 / 3.0)
#define P222 (2.0 / 9.0)

void oracle_set_params(oracle_params *p, int ndte) {
  /* src/ice.F90:80-90 fixed values; :109-130 derived values. */
  const double e_plasticpot = 2.0, e_yieldcurve = 2.0, elasticDamp = 0.36;
  double arlx;
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
  arlx = 2.0 * elasticDamp * (double)ndte;
  p->arlx1i = 1.0 / arlx;
  p->brlx = (double)ndte;
  p->denom1 = 1.0 / (1.0 + p->arlx1i);
  p->deltaminEVP = 10e-9;
}

/* strain_rates (src/bench_v2b.F90:321-397; 2D form src/bench_v0.F90:342-423).
 * Order of the 16 outputs: div ne,nw,sw,se; tension ne,nw,sw,se; shear
 * ne,nw,sw,se; Delta ne,nw,sw,se. */
static inline void strain_rates(double ucc, double vcc, double uee, double vee,
                                double use, double vse, double une, double vne,
                                double dxT, double dyT, double cxp, double cyp,
                                double cxm, double cym, double e_factor,
                                double o[16]) {
  double divune, divunw, divusw, divuse;
  double tne, tnw, tsw, tse, sne, snw, ssw, sse_;
  divune = cyp * ucc - dyT * uee + cxp * vcc - dxT * vse;
  divunw = cym * uee + dyT * ucc + cxp * vee - dxT * vne;
  divusw = cym * une + dyT * use + cxm * vne + dxT * vee;
  divuse = cyp * use - dyT * une + cxm * vse + dxT * vcc;

  tne = -(cym * ucc) - dyT * uee + cxm * vcc + dxT * vse;
  tnw = -(cyp * uee) + dyT * ucc + cxm * vee + dxT * vne;
  tsw = -(cyp * une) + dyT * use + cxp * vne - dxT * vee;
  tse = -(cym * use) - dyT * une + cxp * vse - dxT * vcc;

  sne = -(cym * vcc) - dyT * vee - cxm * ucc - dxT * use;
  snw = -(cyp * vee) + dyT * vcc - cxm * uee - dxT * une;
  ssw = -(cyp * vne) + dyT * vse - cxp * une + dxT * uee;
  sse_ = -(cym * vse) - dyT * vne - cxp * use + dxT * ucc;

  o[0] = divune; o[1] = divunw; o[2] = divusw; o[3] = divuse;
  o[4] = tne; o[5] = tnw; o[6] = tsw; o[7] = tse;
  o[8] = sne; o[9] = snw; o[10] = ssw; o[11] = sse_;
  o[12] = sqrt(divune * divune + e_factor * (tne * tne + sne * sne));
  o[13] = sqrt(divunw * divunw + e_factor * (tnw * tnw + snw * snw));
  o[14] = sqrt(divusw * divusw + e_factor * (tsw * tsw + ssw * ssw));
  o[15] = sqrt(divuse * divuse + e_factor * (tse * tse + sse_ * sse_));
}

/* Fortran MAX(a,b) for non-NaN input. */
static inline double fmax_f(double a, double b) { return a > b ? a : b; }

/* visc_replpress (src/bench_v2b.F90:415-437; v0 :440-470). */
static inline void visc_replpress(double strength, double DminArea,
                                  double Delta, const oracle_params *p,
                                  double *zetax2, double *etax2,
                                  double *rep_prs) {
  double tmpcalc = p->capping * (strength / fmax_f(Delta, DminArea)) +
                   (c1 - p->capping) * (strength / (Delta + DminArea));
  *zetax2 = (c1 + p->Ktens) * tmpcalc;
  *rep_prs = (c1 - p->Ktens) * tmpcalc * Delta;
  *etax2 = p->epp2i * *zetax2;
}

/* The 12 stress updates and the 8 str combinations shared by the v0 and v2
 * kernels (src/bench_v2b.F90:186-310, src/bench_v0.F90:180-329).  s[12] is
 * updated in place; str[8] receives str1..str8. */
static inline void stress_update(double s[12], double out[8], const double sr[16],
                                 double strength, double DminTarea,
                                 double dxt, double dyt, double dxhy,
                                 double dyhx, const oracle_params *p) {
  double zne, znw, zsw, zse, ene, enw, esw, ese, rne, rnw, rsw, rse;
  const double arlx1i = p->arlx1i, denom1 = p->denom1, revp = p->revp;
  const double divune = sr[0], divunw = sr[1], divusw = sr[2], divuse = sr[3];
  const double tne = sr[4], tnw = sr[5], tsw = sr[6], tse = sr[7];
  const double sne = sr[8], snw = sr[9], ssw = sr[10], sse_ = sr[11];
  double ssigpn, ssigps, ssigpe, ssigpw, ssigmn, ssigms, ssigme, ssigmw;
  double ssig12n, ssig12s, ssig12e, ssig12w, ssigp1, ssigp2, ssigm1, ssigm2;
  double ssig121, ssig122, csigpne, csigpnw, csigpse, csigpsw;
  double csigmne, csigmnw, csigmse, csigmsw, csig12ne, csig12nw, csig12se,
      csig12sw;
  double str12ew, str12we, str12ns, str12sn, strp_tmp, strm_tmp;

  visc_replpress(strength, DminTarea, sr[12], p, &zne, &ene, &rne);
  visc_replpress(strength, DminTarea, sr[13], p, &znw, &enw, &rnw);
  visc_replpress(strength, DminTarea, sr[14], p, &zsw, &esw, &rsw);
  visc_replpress(strength, DminTarea, sr[15], p, &zse, &ese, &rse);

  s[0] = (s[0] * (c1 - arlx1i * revp) + arlx1i * (zne * divune - rne)) * denom1;
  s[1] = (s[1] * (c1 - arlx1i * revp) + arlx1i * (znw * divunw - rnw)) * denom1;
  s[2] = (s[2] * (c1 - arlx1i * revp) + arlx1i * (zsw * divusw - rsw)) * denom1;
  s[3] = (s[3] * (c1 - arlx1i * revp) + arlx1i * (zse * divuse - rse)) * denom1;

  s[4] = (s[4] * (c1 - arlx1i * revp) + arlx1i * ene * tne) * denom1;
  s[5] = (s[5] * (c1 - arlx1i * revp) + arlx1i * enw * tnw) * denom1;
  s[6] = (s[6] * (c1 - arlx1i * revp) + arlx1i * esw * tsw) * denom1;
  s[7] = (s[7] * (c1 - arlx1i * revp) + arlx1i * ese * tse) * denom1;

  s[8] = (s[8] * (c1 - arlx1i * revp) + arlx1i * p5 * ene * sne) * denom1;
  s[9] = (s[9] * (c1 - arlx1i * revp) + arlx1i * p5 * enw * snw) * denom1;
  s[10] = (s[10] * (c1 - arlx1i * revp) + arlx1i * p5 * esw * ssw) * denom1;
  s[11] = (s[11] * (c1 - arlx1i * revp) + arlx1i * p5 * ese * sse_) * denom1;

  ssigpn = s[0] + s[1];
  ssigps = s[2] + s[3];
  ssigpe = s[0] + s[3];
  ssigpw = s[1] + s[2];
  ssigp1 = (s[0] + s[2]) * P055;
  ssigp2 = (s[1] + s[3]) * P055;

  ssigmn = s[4] + s[5];
  ssigms = s[6] + s[7];
  ssigme = s[4] + s[7];
  ssigmw = s[5] + s[6];
  ssigm1 = (s[4] + s[6]) * P055;
  ssigm2 = (s[5] + s[7]) * P055;

  ssig12n = s[8] + s[9];
  ssig12s = s[10] + s[11];
  ssig12e = s[8] + s[11];
  ssig12w = s[9] + s[10];
  ssig121 = (s[8] + s[10]) * P111;
  ssig122 = (s[9] + s[11]) * P111;

  csigpne = P111 * s[0] + ssigp2 + P027 * s[2];
  csigpnw = P111 * s[1] + ssigp1 + P027 * s[3];
  csigpsw = P111 * s[2] + ssigp2 + P027 * s[0];
  csigpse = P111 * s[3] + ssigp1 + P027 * s[1];

  csigmne = P111 * s[4] + ssigm2 + P027 * s[6];
  csigmnw = P111 * s[5] + ssigm1 + P027 * s[7];
  csigmsw = P111 * s[6] + ssigm2 + P027 * s[4];
  csigmse = P111 * s[7] + ssigm1 + P027 * s[5];

  csig12ne = P222 * s[8] + ssig122 + P055 * s[10];
  csig12nw = P222 * s[9] + ssig121 + P055 * s[11];
  csig12sw = P222 * s[10] + ssig122 + P055 * s[8];
  csig12se = P222 * s[11] + ssig121 + P055 * s[9];

  str12ew = p5 * dxt * (P333 * ssig12e + P166 * ssig12w);
  str12we = p5 * dxt * (P333 * ssig12w + P166 * ssig12e);
  str12ns = p5 * dyt * (P333 * ssig12n + P166 * ssig12s);
  str12sn = p5 * dyt * (P333 * ssig12s + P166 * ssig12n);

  strp_tmp = p25 * dyt * (P333 * ssigpn + P166 * ssigps);
  strm_tmp = p25 * dyt * (P333 * ssigmn + P166 * ssigms);
  out[0] = -strp_tmp - strm_tmp - str12ew + dxhy * (-csigpne + csigmne) +
           dyhx * csig12ne;
  out[1] = strp_tmp + strm_tmp - str12we + dxhy * (-csigpnw + csigmnw) +
           dyhx * csig12nw;

  strp_tmp = p25 * dyt * (P333 * ssigps + P166 * ssigpn);
  strm_tmp = p25 * dyt * (P333 * ssigms + P166 * ssigmn);
  out[2] = -strp_tmp - strm_tmp + str12ew + dxhy * (-csigpse + csigmse) +
           dyhx * csig12se;
  out[3] = strp_tmp + strm_tmp + str12we + dxhy * (-csigpsw + csigmsw) +
           dyhx * csig12sw;

  strp_tmp = p25 * dxt * (P333 * ssigpe + P166 * ssigpw);
  strm_tmp = p25 * dxt * (P333 * ssigme + P166 * ssigmw);
  out[4] = -strp_tmp + strm_tmp - str12ns - dyhx * (csigpne + csigmne) +
           dxhy * csig12ne;
  out[5] = strp_tmp - strm_tmp - str12sn - dyhx * (csigpse + csigmse) +
           dxhy * csig12se;

  strp_tmp = p25 * dxt * (P333 * ssigpw + P166 * ssigpe);
  strm_tmp = p25 * dxt * (P333 * ssigmw + P166 * ssigme);
  out[6] = -strp_tmp + strm_tmp + str12ns - dyhx * (csigpnw + csigmnw) +
           dxhy * csig12nw;
  out[7] = strp_tmp - strm_tmp + str12sn - dyhx * (csigpsw + csigmsw) +
           dxhy * csig12sw;
}

/* ------------------------------------------------------------------------ */
/* v2b 1D stress: src/bench_v2b.F90:62-312                                   */
/* ------------------------------------------------------------------------ */
void oracle_stress_1d(const int32_t *ee, const int32_t *ne, const int32_t *se,
                      int lb, int ub, const double *uvel, const double *vvel,
                      const double *dxT, const double *dyT,
                      const int32_t *skipme, const double *strength,
                      const double *hte, const double *htn,
                      const double *htem1, const double *htnm1,
                      double *const stress[12], double *const str[8],
                      const oracle_params *p) {
  int iw, k;
  for (iw = lb; iw <= ub; iw++) {
    const int w = iw - 1;
    double sr[16], s[12], out[8];
    double ucc, vcc, uee, vse, vee, vne, une, use, tdxT, tdyT;
    double cxp, cyp, cxm, cym, tmparea, DminTarea, dxhy, dyhx;
    if (skipme[w]) continue;
    ucc = uvel[w];
    vcc = vvel[w];
    uee = uvel[ee[w] - 1];
    vse = vvel[se[w] - 1];
    vee = vvel[ee[w] - 1];
    vne = vvel[ne[w] - 1];
    une = uvel[ne[w] - 1];
    use = uvel[se[w] - 1];
    tdxT = dxT[w];
    tdyT = dyT[w];
    /* geometry derivation, src/bench_v2b.F90:139-147 */
    cxp = c1p5 * htn[w] - p5 * htnm1[w];
    cyp = c1p5 * hte[w] - p5 * htem1[w];
    cxm = -(c1p5 * htnm1[w] - p5 * htn[w]);
    cym = -(c1p5 * htem1[w] - p5 * hte[w]);
    tmparea = dxT[w] * dyT[w];
    DminTarea = p->deltaminEVP * tmparea;
    dxhy = p5 * (hte[w] - htem1[w]);
    dyhx = p5 * (htn[w] - htnm1[w]);
    strain_rates(ucc, vcc, uee, vee, use, vse, une, vne, tdxT, tdyT, cxp, cyp,
                 cxm, cym, p->e_factor, sr);
    for (k = 0; k < 12; k++) s[k] = stress[k][w];
    stress_update(s, out, sr, strength[w], DminTarea, tdxT, tdyT, dxhy, dyhx,
                  p);
    for (k = 0; k < 12; k++) stress[k][w] = s[k];
    for (k = 0; k < 8; k++) str[k][w] = out[k];
  }
}

/* ------------------------------------------------------------------------ */
/* v2b 1D stepu: src/bench_v2b.F90:444-549                                   */
/* ------------------------------------------------------------------------ */
void oracle_stepu_1d(int lb, int ub, const double *Cw, const double *aiX,
                     const double *uocn, const double *vocn,
                     const double *waterx, const double *watery,
                     const double *forcex, const double *forcey,
                     const double *umassdti, const double *fm,
                     const double *uarear, double *strintx, double *strinty,
                     const double *uvel_init, const double *vvel_init,
                     double *uvel, double *vvel, double *const str[8],
                     const int32_t *nw, const int32_t *sw, const int32_t *sse,
                     const int32_t *skipme, const double *Tbu, double *Cb,
                     const oracle_params *p) {
  const double rhow = p->rhow, brlx = p->brlx, revp = p->revp, u0 = p->u0;
  const double cosw = p->cosw, sinw = p->sinw;
  int iw;
  for (iw = lb; iw <= ub; iw++) {
    const int w = iw - 1;
    double uold, vold, vrel, taux, tauy, cca, ccb, ab2, cc1, cc2;
    double s2nw, s3sse, s4sw, s6sse, s7nw, s8sw;
    if (skipme[w]) continue;
    uold = uvel[w];
    vold = vvel[w];
    vrel = aiX[w] * rhow * Cw[w] *
           sqrt((uocn[w] - uold) * (uocn[w] - uold) +
                (vocn[w] - vold) * (vocn[w] - vold));
    taux = vrel * waterx[w];
    tauy = vrel * watery[w];
    Cb[w] = Tbu[w] / (sqrt(uold * uold + vold * vold) + u0);
    cca = (brlx + revp) * umassdti[w] + vrel * cosw + Cb[w];
    ccb = fm[w] + copysign(c1, fm[w]) * vrel * sinw;
    ab2 = cca * cca + ccb * ccb;
    s2nw = str[1][nw[w] - 1];
    s3sse = str[2][sse[w] - 1];
    s4sw = str[3][sw[w] - 1];
    s6sse = str[5][sse[w] - 1];
    s7nw = str[6][nw[w] - 1];
    s8sw = str[7][sw[w] - 1];
    strintx[w] = uarear[w] * (str[0][w] + s2nw + s3sse + s4sw);
    strinty[w] = uarear[w] * (str[4][w] + s6sse + s7nw + s8sw);
    cc1 = strintx[w] + forcex[w] + taux +
          umassdti[w] * (brlx * uold + revp * uvel_init[w]);
    cc2 = strinty[w] + forcey[w] + tauy +
          umassdti[w] * (brlx * vold + revp * vvel_init[w]);
    uvel[w] = (cca * cc1 + ccb * cc2) / ab2;
    vvel[w] = (cca * cc2 - ccb * cc1) / ab2;
  }
}

#define STRESS_ARGS(s, lb, ub)                                                 \
  (s)->ee, (s)->ne, (s)->se, (lb), (ub), (s)->uvel, (s)->vvel, (s)->dxT,       \
      (s)->dyT, (s)->skipT, (s)->strength, (s)->HTE, (s)->HTN, (s)->HTEm1,     \
      (s)->HTNm1, (s)->stress, (s)->str
#define STEPU_ARGS(s, lb, ub)                                                  \
  (lb), (ub), (s)->Cw, (s)->aiu, (s)->uocn, (s)->vocn, (s)->waterx,            \
      (s)->watery, (s)->forcex, (s)->forcey, (s)->umassdti, (s)->fm,           \
      (s)->uarear, (s)->strintx, (s)->strinty, (s)->uvel_init,                 \
      (s)->vvel_init, (s)->uvel, (s)->vvel, (s)->str, (s)->nw, (s)->sw,        \
      (s)->sse, (s)->skipU, (s)->Tbu, (s)->Cb

/* integration/ice_dyn_evp1d.F90:188-207 */
void oracle_run_1d(oracle_1d *s, int ndte, const oracle_params *p) {
  int k;
  for (k = 0; k < ndte; k++) {
    oracle_stress_1d(STRESS_ARGS(s, 1, s->na), p);
    oracle_stepu_1d(STEPU_ARGS(s, 1, s->na), p);
  }
}

/* src/evp_v2b.F90:127-141 */
void oracle_stress_only_1d(oracle_1d *s, int n, const oracle_params *p) {
  int k;
  for (k = 0; k < n; k++) oracle_stress_1d(STRESS_ARGS(s, 1, s->na), p);
}

/* src/evp_v2b.F90:143-153 */
void oracle_stepu_only_1d(oracle_1d *s, int n, const oracle_params *p) {
  int k;
  for (k = 0; k < n; k++) oracle_stepu_1d(STEPU_ARGS(s, 1, s->na), p);
}

/* myomp:domp_get_domain_rlu (src/myomp.F90:85-124). */
void oracle_omp_domain(int lower, int upper, int iam, int nt, int *dl,
                       int *du) {
  double dlen;
  if (upper <= 0 || upper < lower) {
    *dl = 0;
    *du = -1;
    return;
  }
  if (nt <= 1) {
    *dl = lower;
    *du = upper;
    return;
  }
  dlen = (double)(upper - lower + 1);
  *dl = lower + (int)floor(((double)iam * dlen + p5) / (double)nt);
  *du = lower - 1 + (int)floor(((double)iam * dlen + dlen + p5) / (double)nt);
}

/* src/evp_v2b.F90:91-110: !$OMP PARALLEL; do ndte: stress; barrier; stepu;
 * barrier. */
int oracle_run_1d_omp(oracle_1d *s, int ndte, const oracle_params *p,
                      int nthreads) {
  int used = 1;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    int il, iu, k;
    const int iam = omp_get_thread_num(), nt = omp_get_num_threads();
#pragma omp single
    used = nt;
    oracle_omp_domain(1, s->na, iam, nt, &il, &iu);
    for (k = 0; k < ndte; k++) {
      if (iu >= il) oracle_stress_1d(STRESS_ARGS(s, il, iu), p);
#pragma omp barrier
      if (iu >= il) oracle_stepu_1d(STEPU_ARGS(s, il, iu), p);
#pragma omp barrier
    }
  }
#else
  (void)nthreads;
  oracle_run_1d(s, ndte, p);
#endif
  return used;
}

void oracle_first_touch_1d(double *buf, long n, int nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    int dl, du;
    const int iam = omp_get_thread_num(), nt = omp_get_num_threads();
    oracle_omp_domain(1, (int)n, iam, nt, &dl, &du);
    if (du >= dl) memset(buf + (dl - 1), 0, sizeof(double) * (size_t)(du - dl + 1));
  }
#else
  (void)nthreads;
  memset(buf, 0, sizeof(double) * (size_t)n);
#endif
}

/* ------------------------------------------------------------------------ */
/* v0 2D kernels: src/bench_v0.F90                                           */
/* ------------------------------------------------------------------------ */
#define IX(i, j) ((size_t)((i) - 1) + (size_t)((j) - 1) * (size_t)nxb)

/* stress: src/bench_v0.F90:50-333 */
void oracle_stress_2d(int nxb, int nyb, int icellt, const int32_t *indxti,
                      const int32_t *indxtj, const double *uvel,
                      const double *vvel, const double *dxT,
                      const double *dyT, const double *dxhy,
                      const double *dyhx, const double *cxp,
                      const double *cyp, const double *cxm, const double *cym,
                      const double *DminTarea, const double *strength,
                      double *const stress[12], double *str,
                      const oracle_params *p) {
  const size_t plane = (size_t)nxb * (size_t)nyb;
  int ij, k;
  memset(str, 0, sizeof(double) * plane * 8); /* str(:,:,:) = c0, :132 */
  for (ij = 0; ij < icellt; ij++) {
    const int i = indxti[ij], j = indxtj[ij];
    const size_t c = IX(i, j);
    double sr[16], s[12], out[8];
    /* uvel(i-1,j)=ee, uvel(i-1,j-1)=ne, uvel(i,j-1)=se (:389-416) */
    strain_rates(uvel[c], vvel[c], uvel[IX(i - 1, j)], vvel[IX(i - 1, j)],
                 uvel[IX(i, j - 1)], vvel[IX(i, j - 1)],
                 uvel[IX(i - 1, j - 1)], vvel[IX(i - 1, j - 1)], dxT[c],
                 dyT[c], cxp[c], cyp[c], cxm[c], cym[c], p->e_factor, sr);
    for (k = 0; k < 12; k++) s[k] = stress[k][c];
    stress_update(s, out, sr, strength[c], DminTarea[c], dxT[c], dyT[c],
                  dxhy[c], dyhx[c], p);
    for (k = 0; k < 12; k++) stress[k][c] = s[k];
    for (k = 0; k < 8; k++) str[c + (size_t)k * plane] = out[k];
  }
}

/* stepu: src/bench_v0.F90:478-603 */
void oracle_stepu_2d(int nxb, int nyb, int icellu, const double *Cw,
                     const int32_t *indxui, const int32_t *indxuj,
                     const double *aiX, const double *str, const double *uocn,
                     const double *vocn, const double *waterx,
                     const double *watery, const double *forcex,
                     const double *forcey, const double *umassdti,
                     const double *fm, const double *uarear, double *strintx,
                     double *strinty, double *taubx, double *tauby,
                     const double *uvel_init, const double *vvel_init,
                     double *uvel, double *vvel, const double *Tbu,
                     const oracle_params *p) {
  const size_t plane = (size_t)nxb * (size_t)nyb;
  const double rhow = p->rhow, brlx = p->brlx, revp = p->revp, u0 = p->u0;
  const double cosw = p->cosw, sinw = p->sinw;
  int ij;
#define STR(i, j, k) str[IX(i, j) + (size_t)((k) - 1) * plane]
  for (ij = 0; ij < icellu; ij++) {
    const int i = indxui[ij], j = indxuj[ij];
    const size_t c = IX(i, j);
    double uold, vold, vrel, taux, tauy, Cb, cca, ccb, ab2, cc1, cc2;
    uold = uvel[c];
    vold = vvel[c];
    vrel = aiX[c] * rhow * Cw[c] *
           sqrt((uocn[c] - uold) * (uocn[c] - uold) +
                (vocn[c] - vold) * (vocn[c] - vold));
    taux = vrel * waterx[c];
    tauy = vrel * watery[c];
    Cb = Tbu[c] / (sqrt(uold * uold + vold * vold) + u0);
    cca = (brlx + revp) * umassdti[c] + vrel * cosw + Cb;
    ccb = fm[c] + copysign(c1, fm[c]) * vrel * sinw;
    ab2 = cca * cca + ccb * ccb;
    strintx[c] = uarear[c] * (STR(i, j, 1) + STR(i + 1, j, 2) +
                              STR(i, j + 1, 3) + STR(i + 1, j + 1, 4));
    strinty[c] = uarear[c] * (STR(i, j, 5) + STR(i, j + 1, 6) +
                              STR(i + 1, j, 7) + STR(i + 1, j + 1, 8));
    cc1 = strintx[c] + forcex[c] + taux +
          umassdti[c] * (brlx * uold + revp * uvel_init[c]);
    cc2 = strinty[c] + forcey[c] + tauy +
          umassdti[c] * (brlx * vold + revp * vvel_init[c]);
    uvel[c] = (cca * cc1 + ccb * cc2) / ab2;
    vvel[c] = (cca * cc2 - ccb * cc1) / ab2;
    taubx[c] = -uvel[c] * Cb;
    tauby[c] = -vvel[c] * Cb;
  }
#undef STR
}

/* ------------------------------------------------------------------------ */
/* evp1d adapter index build                                                 */
/* ------------------------------------------------------------------------ */

/* union of two sorted vectors (integration/ice_dyn_evp1d.F90:591-633). */
static int sorted_union(const int32_t *x, int nxv, const int32_t *y, int nyv,
                        int32_t *xy) {
  int i = 0, j = 0, k = 0;
  while (i < nxv && j < nyv) {
    if (x[i] < y[j]) xy[k++] = x[i++];
    else if (x[i] > y[j]) xy[k++] = y[j++];
    else { xy[k++] = x[i++]; j++; }
  }
  while (i < nxv) xy[k++] = x[i++];
  while (j < nyv) xy[k++] = y[j++];
  return k;
}

/* symmetric difference of two sorted vectors (:951-998). */
static int sorted_setdiff(const int32_t *x, int nxv, const int32_t *y, int nyv,
                          int32_t *xy) {
  int i = 0, j = 0, k = 0;
  while (i < nxv && j < nyv) {
    if (x[i] < y[j]) xy[k++] = x[i++];
    else if (x[i] > y[j]) xy[k++] = y[j++];
    else { i++; j++; }
  }
  while (i < nxv) xy[k++] = x[i++];
  while (j < nyv) xy[k++] = y[j++];
  return k;
}

/* findXinY (:1000-1045): x sorted; y = [sorted y(1:nx) ; sorted y(nx+1:ny)].
 * Writes 1-based positions.  Returns -2 where the reference stops. */
static int find_x_in_y(const int32_t *x, int nxv, const int32_t *y, int nyv,
                       int32_t *indx) {
  int i = 0, j1 = 0, j2 = nxv;
  while (i < nxv) {
    if (j1 >= nyv && j2 >= nyv) return -2;
    if (j1 < nyv && x[i] == y[j1]) { indx[i] = j1 + 1; i++; j1++; }
    else if (j2 < nyv && x[i] == y[j2]) { indx[i] = j2 + 1; i++; j2++; }
    else if (j1 < nyv && x[i] > y[j1]) j1++;
    else if (j2 < nyv && x[i] > y[j2]) j2++;
    else return -2;
  }
  return 0;
}

int oracle_build_index(int nx, int ny, int nghost, const int32_t *mask,
                       int cap_na, int cap_navel, int *na_out,
                       int *navel_out, int32_t *indxti, int32_t *indxtj,
                       int32_t *indxtij, int32_t *ee, int32_t *ne,
                       int32_t *se, int32_t *nw, int32_t *sw, int32_t *sse) {
  int i, j, na = 0, n1, n2, nh, k, rc = 0;
  int32_t *off[7], *u1 = NULL, *u2 = NULL;
  int32_t *outs[6];
  /* calc_2d_indices_init (:559-589): j outer, i inner, from 1+nghost. */
  for (j = 1 + nghost; j <= ny; j++)
    for (i = 1 + nghost; i <= nx; i++)
      if (mask[(size_t)(i - 1) + (size_t)(j - 1) * (size_t)nx]) {
        if (na >= cap_na) return -1;
        indxti[na] = i;
        indxtj[na] = j;
        na++;
      }
  *na_out = na;
  for (k = 0; k < 7; k++) {
    off[k] = (int32_t *)malloc(sizeof(int32_t) * (size_t)(na > 0 ? na : 1));
  }
  u1 = (int32_t *)malloc(sizeof(int32_t) * (size_t)(7 * (na > 0 ? na : 1)));
  u2 = (int32_t *)malloc(sizeof(int32_t) * (size_t)(7 * (na > 0 ? na : 1)));
  /* linear indices of the 7 stencil offsets (:761-773). */
  for (k = 0; k < na; k++) {
    i = indxti[k];
    j = indxtj[k];
    off[0][k] = i + (j - 1) * nx;     /* ( 0, 0) */
    off[1][k] = i - 1 + (j - 1) * nx; /* (-1, 0) ee  */
    off[2][k] = i - 1 + (j - 2) * nx; /* (-1,-1) ne  */
    off[3][k] = i + (j - 2) * nx;     /* ( 0,-1) se  */
    off[4][k] = i + 1 + (j - 1) * nx; /* (+1, 0) nw  */
    off[5][k] = i + 1 + (j - 0) * nx; /* (+1,+1) sw  */
    off[6][k] = i + (j - 0) * nx;     /* ( 0,+1) sse */
  }
  /* union chain (:775-780) */
  n1 = sorted_union(off[0], na, off[1], na, u1);
  n2 = sorted_union(u1, n1, off[2], na, u2);
  n1 = sorted_union(u2, n2, off[3], na, u1);
  n2 = sorted_union(u1, n1, off[4], na, u2);
  n1 = sorted_union(u2, n2, off[5], na, u1);
  n2 = sorted_union(u1, n1, off[6], na, u2); /* navel */
  *navel_out = n2;
  if (n2 > cap_navel) { rc = -1; goto done; }
  for (k = 0; k < na; k++) indxtij[k] = off[0][k];
  nh = sorted_setdiff(u2, n2, off[0], na, u1); /* halo, sorted (:786-790) */
  for (k = 0; k < nh; k++) indxtij[na + k] = u1[k];
  outs[0] = ee; outs[1] = ne; outs[2] = se;
  outs[3] = nw; outs[4] = sw; outs[5] = sse;
  for (k = 0; k < 6; k++) {
    if (find_x_in_y(off[k + 1], na, indxtij, n2, outs[k]) != 0) {
      rc = -2;
      goto done;
    }
  }
done:
  for (k = 0; k < 7; k++) free(off[k]);
  free(u1);
  free(u2);
  return rc;
}
