/*
 * EVP-1D ORACLE -- test infrastructure only.
 *
 * A plain-C, CPU-only restatement of the reference's EVP arithmetic
 * (dmidk/cice-evp1d), used as the checker for the CUDA path:
 *   - the v0 upstream 2D kernels   (src/bench_v0.F90:50-603),
 *   - the v2b 1D kernels           (src/bench_v2b.F90:62-549),
 *   - the evp1d adapter index build (integration/ice_dyn_evp1d.F90:559-589,
 *     591-633, 743-816, 951-1087),
 *   - the v2b SPMD OpenMP driver loop with the myomp static split
 *     (src/evp_v2b.F90:91-110, src/myomp.F90:85-124), timed as the CPU
 *     baseline.
 *
 * Every expression keeps the Fortran evaluation order (left to right within
 * one precedence level, parentheses honoured, x**2 as x*x, sign() as
 * copysign).  Built with -ffp-contract=off -fno-fast-math this matches the
 * reference's f0/f1 (-fp-model precise -no-fma) semantics.
 *
 * Parity unpinned against the reference's own outputs: its only golden
 * vectors are md5 sums over DMI input files that are not distributed
 * (README.md:63-104), and the Fortran reference cannot be compiled in this
 * image.  The oracle is held instead by the reference's own acceptance
 * criterion -- the v0 2D form and the v2 1D form produce md5-identical output
 * files on the same input -- by closed-form answers of the integration smoke
 * test state (integration/ice_dyn_evp1d_standalone.F90:60-79), and by the
 * committed fixture in tests/golden.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline may use
 * this code.  The product path never links it.
 */
#ifndef EVP_ORACLE_H
#define EVP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* EVP parameters; the fields and their meaning follow src/ice.F90:80-130
 * (set_evp_parameters) and the input overrides of src/vars.F90:2116. */
typedef struct {
  double arlx1i, denom1, brlx;
  double capping, e_factor, epp2i, deltaminEVP;
  double revp, Ktens;
  double u0, cosw, sinw, rhow;
} oracle_params;

/* set_evp_parameters(dt) for a given ndte (src/ice.F90:109-130). */
void oracle_set_params(oracle_params *p, int ndte);

/* ---------------- v2b 1D kernels (1-based neighbour indices) -------------- */
/* stress(ee,ne,se,lb,ub, uvel,vvel,dxT,dyT,skipme,strength,hte,htn,htem1,htnm1,
 *        12 stresses, str1..str8)  src/bench_v2b.F90:62-312.
 * lb, ub are 1-based inclusive bounds.  stress[0..11] = stressp_1..4,
 * stressm_1..4, stress12_1..4.  str[0..7] = str1..str8. */
void oracle_stress_1d(const int32_t *ee, const int32_t *ne, const int32_t *se,
                      int lb, int ub, const double *uvel, const double *vvel,
                      const double *dxT, const double *dyT,
                      const int32_t *skipme, const double *strength,
                      const double *hte, const double *htn,
                      const double *htem1, const double *htnm1,
                      double *const stress[12], double *const str[8],
                      const oracle_params *p);

/* stepu(lb,ub, Cw,aiX,uocn,vocn,waterx,watery,forcex,forcey,umassdti,fm,
 *       uarear, strintx,strinty, uvel_init,vvel_init, uvel,vvel, str1..8,
 *       nw,sw,sse,skipme, Tbu,Cb)   src/bench_v2b.F90:444-549. */
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
                     const oracle_params *p);

/* The 1D problem in the reference's v2 layout (all arrays 0-based in C,
 * neighbour indices 1-based as in Fortran, navel-sized arrays for u, v, str).
 */
typedef struct {
  int na, navel;
  const int32_t *ee, *ne, *se, *nw, *sw, *sse; /* [na], 1-based */
  const int32_t *skipT, *skipU;                /* [na], 0/1 */
  const double *dxT, *dyT, *HTE, *HTN, *HTEm1, *HTNm1, *strength; /* [na] */
  const double *Cw, *aiu, *uocn, *vocn, *waterx, *watery, *forcex, *forcey;
  const double *umassdti, *fm, *uarear, *Tbu, *uvel_init, *vvel_init;
  double *stress[12];  /* [na]    inout */
  double *uvel, *vvel; /* [navel] inout */
  double *str[8];      /* [navel] inout (scratch; starts at 0) */
  double *strintx, *strinty, *Cb; /* [na] inout */
} oracle_1d;

/* Serial subcycle loop: ndte x { stress(1..na); stepu(1..na) }
 * (integration/ice_dyn_evp1d.F90:188-207). */
void oracle_run_1d(oracle_1d *s, int ndte, const oracle_params *p);
/* lindividual-style loops (src/evp_v2b.F90:127-155). */
void oracle_stress_only_1d(oracle_1d *s, int n, const oracle_params *p);
void oracle_stepu_only_1d(oracle_1d *s, int n, const oracle_params *p);

/* SPMD OpenMP loop with the myomp static split and a barrier after each phase
 * (src/evp_v2b.F90:91-110).  nthreads <= 0 means the OpenMP default.
 * Returns the thread count used (1 when built without OpenMP). */
int oracle_run_1d_omp(oracle_1d *s, int ndte, const oracle_params *p,
                      int nthreads);
/* myomp:domp_get_domain static split for thread `iam` of `nt`
 * (src/myomp.F90:85-124); bounds 1-based inclusive. */
void oracle_omp_domain(int lower, int upper, int iam, int nt, int *dl,
                       int *du);
/* First-touch zeroing of every array of the problem, per thread slice
 * (src/numa.F90:144-223).  Used by the CPU baseline before timing. */
void oracle_first_touch_1d(double *buf, long n, int nthreads);

/* ---------------- v0 2D kernels (Fortran column-major, 1-based) ----------- */
/* Arrays are [nxb*nyb] with element (i,j) at (i-1)+(j-1)*nxb.  str is
 * [nxb*nyb*8] (str(i,j,k) at (i-1)+(j-1)*nxb+(k-1)*nxb*nyb). */
void oracle_stress_2d(int nxb, int nyb, int icellt, const int32_t *indxti,
                      const int32_t *indxtj, const double *uvel,
                      const double *vvel, const double *dxT,
                      const double *dyT, const double *dxhy,
                      const double *dyhx, const double *cxp,
                      const double *cyp, const double *cxm, const double *cym,
                      const double *DminTarea, const double *strength,
                      double *const stress[12], double *str,
                      const oracle_params *p);
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
                     const oracle_params *p);

/* ---------------- evp1d adapter index build -------------------------------- */
/* calc_2d_indices_init + calc_navel + convert_2d_1d_init index part
 * (integration/ice_dyn_evp1d.F90:559-589, 743-797, 1047-1087).
 * mask is [nx*ny] column-major (i fastest), nonzero = active.
 * Outputs (caller-allocated): indxti, indxtj [cap_na] (1-based i,j);
 * indxtij [cap_navel] (1-based linear index i+(j-1)*nx);
 * ee,ne,se,nw,sw,sse [cap_na] 1-based into 1..navel.
 * Returns 0, -1 if a capacity is too small, -2 if a neighbour is not found
 * (the reference stops there, :1039). */
int oracle_build_index(int nx, int ny, int nghost, const int32_t *mask,
                       int cap_na, int cap_navel, int *na_out,
                       int *navel_out, int32_t *indxti, int32_t *indxtj,
                       int32_t *indxtij, int32_t *ee, int32_t *ne,
                       int32_t *se, int32_t *nw, int32_t *sw, int32_t *sse);

#ifdef __cplusplus
}
#endif
#endif
