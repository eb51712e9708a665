/*
 * evp1d.h -- C-ABI of the B200 (sm_100a) EVP-1D sea-ice dynamics solver.
 *
 * Drop-in for the ndte-subcycle loop of CICE's 1D EVP solver as restructured
 * by dmidk/cice-evp1d: the `stress` and `stepu` kernels of module `bench`
 * (src/bench_v2b.F90:62-312, 444-549) called ndte times from
 * dyn_evp1d_run (integration/ice_dyn_evp1d.F90:188-207).
 *
 * Conventions
 *  - Plain C types only: int32_t indices, double fields, host pointers unless
 *    a function says "device".
 *  - 1D layout as in the reference: `na` list points, `navel >= na` slots
 *    where slots na+1..navel are halo points (outside the list).  Neighbour
 *    vectors are 1-BASED, exactly as the Fortran module stores them
 *    (integration/ice_dyn_evp1d.F90:792-797).  Per-point fields have length
 *    na; uvel, vvel and str1..str8 have length navel.
 *  - Every function returns EVP1D_OK (0) or a negative EVP1D_ERR_* code;
 *    evp1d_last_error() gives a message.  Nothing aborts the process (the
 *    reference calls `stop`, integration/ice_dyn_evp1d.F90:394-460,1039).
 *  - A handle owns its device buffers and one CUDA stream.  It is not
 *    thread-safe; use one handle per host thread.
 *  - All arithmetic is IEEE FP64 in the reference's operation order with no
 *    FMA contraction: results are bit-identical to the reference's f0/f1
 *    (-fp-model precise -no-fma) builds on the same input.
 */
#ifndef EVP1D_H
#define EVP1D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EVP1D_OK 0
#define EVP1D_ERR_INVALID_ARG (-1) /* NULL pointer, bad size, bad ndte       */
#define EVP1D_ERR_INDEX (-2)       /* neighbour index outside 1..navel, or a
                                      list point that is not its own slot   */
#define EVP1D_ERR_CUDA (-3)        /* a CUDA runtime call failed            */
#define EVP1D_ERR_NOMEM (-4)       /* device or pinned allocation failed    */
#define EVP1D_ERR_TIMEOUT (-5)     /* a bounded device-side wait ran out    */
#define EVP1D_ERR_NO_DEVICE (-6)   /* no CUDA device of compute 10.x        */
#define EVP1D_ERR_STATE (-7)       /* call out of order (e.g. no upload)    */

/* EVP parameters.  Field meanings follow ice_dyn_shared (src/ice.F90:80-130)
 * including the values read from the input file (src/vars.F90:2116). */
typedef struct evp1d_params {
  double arlx1i;      /* 1 / (2 * elasticDamp * ndte)                   */
  double denom1;      /* 1 / (1 + arlx1i)                               */
  double brlx;        /* ndte                                           */
  double capping;     /* 1: capped viscosities                          */
  double e_factor;    /* e_yieldcurve^2 / e_plasticpot^4                */
  double epp2i;       /* 1 / e_plasticpot^2                             */
  double deltaminEVP; /* minimum Delta (1e-8)                           */
  double revp;        /* 0 classic EVP, 1 revised EVP                   */
  double Ktens;       /* tensile strength factor                        */
  double u0;          /* basal-stress residual speed (5e-5 m/s)         */
  double cosw, sinw;  /* ocean turning angle                            */
  double rhow;        /* sea-water density (1026 kg/m^3)                */
} evp1d_params;

/* Per-call fields of dyn_evp1d_run in the 1D layout (host pointers).
 * Replaces the argument lists of stress/stepu (src/bench_v2b.F90:62-68,
 * 444-458) and the L_* arrays of dyn_evp1d_run
 * (integration/ice_dyn_evp1d.F90:115-138).  in = read, inout = read and
 * written back, out = written. */
typedef struct evp1d_fields {
  const int32_t *skipT;     /* in  [na]  nonzero: not an ice T point      */
  const int32_t *skipU;     /* in  [na]  nonzero: not an ice U point      */
  double *stress[12];       /* inout [na] stressp_1..4, stressm_1..4,
                                          stress12_1..4                  */
  const double *strength;   /* in  [na]                                   */
  const double *Cw;         /* in  [na]  cdn_ocn                          */
  const double *aiu;        /* in  [na]                                   */
  const double *uocn, *vocn;      /* in [na]                              */
  const double *waterx, *watery;  /* in [na]                              */
  const double *forcex, *forcey;  /* in [na]                              */
  const double *umassdti;   /* in  [na]                                   */
  const double *fm;         /* in  [na]                                   */
  const double *Tbu;        /* in  [na]                                   */
  const double *uvel_init;  /* in  [na]  NULL: uvel at the start of the call
                                         (src/vars.F90:2119-2120)         */
  const double *vvel_init;  /* in  [na]  NULL: vvel at the start          */
  double *uvel, *vvel;      /* inout [navel]; list slots 1..na are updated,
                               halo slots na+1..navel are read as given and
                               never written (the adapter passes 0 there,
                               integration/ice_dyn_evp1d.F90:880-881)      */
  double *strintx, *strinty;/* inout [na]; written at ice U points        */
  double *Cb;               /* inout [na]; written at ice U points        */
  double *str[8];           /* out [navel] str1..str8 of the last subcycle,
                               each may be NULL (not returned)            */
} evp1d_fields;

typedef struct evp1d_handle evp1d_t;

/* set_evp_parameters for a given ndte (src/ice.F90:109-130). */
void evp1d_set_evp_parameters(evp1d_params *p, int ndte);

/* Set up the static part of the 1D problem on `device`.
 * Replaces the index/geometry part of dyn_evp1d_init
 * (integration/ice_dyn_evp1d.F90:65-112, 743-816): neighbour vectors (1-based,
 * [na]) and the static per-point geometry ([na]).  Indices are validated on
 * the host (EVP1D_ERR_INDEX) so that no device access can leave its buffer.
 * na = 0 is allowed (every run is then a no-op). */
int evp1d_init(evp1d_t **handle, int na, int navel, const int32_t *ee,
               const int32_t *ne, const int32_t *se, const int32_t *nw,
               const int32_t *sw, const int32_t *sse, const double *dxT,
               const double *dyT, const double *HTE, const double *HTN,
               const double *HTEm1, const double *HTNm1, const double *uarear,
               const evp1d_params *params, int device);

/* An ensemble of independent 1D problems (members) solved together: one
 * tile plan over all members, one kernel launch per subcycle for the whole
 * ensemble.  Member m has na[m] list points and navel[m] slots; its neighbour
 * vectors are 1-based within the member.  Every array argument here and in
 * the evp1d_fields of later calls is the member-major concatenation of the
 * members' arrays (per-point fields: sum(na) entries; uvel, vvel, str:
 * sum(navel) entries, each member's halo slots after its own list points).
 * Results are bitwise those of solving each member alone.  No counterpart in
 * the reference, which solves one state per call. */
int evp1d_init_batched(evp1d_t **handle, int nmembers, const int32_t *na,
                       const int32_t *navel, const int32_t *ee,
                       const int32_t *ne, const int32_t *se, const int32_t *nw,
                       const int32_t *sw, const int32_t *sse,
                       const double *dxT, const double *dyT, const double *HTE,
                       const double *HTN, const double *HTEm1,
                       const double *HTNm1, const double *uarear,
                       const evp1d_params *params, int device);

/* Time the kernel variants (TMA-fed with and without L2 prefetch, plain
 * loads) for `nsub` subcycles on the uploaded state, keep the fastest for
 * this handle and restore the state.  `chosen` (may be NULL) receives a
 * description of the choice.  Needs a prior evp1d_upload. */
int evp1d_autotune(evp1d_t *handle, int nsub, char *chosen, int len);

/* Release the handle and its device buffers (dyn_evp1d_finalize,
 * integration/ice_dyn_evp1d.F90:326-331).  NULL is a no-op. */
int evp1d_finalize(evp1d_t *handle);

/* Replace the EVP parameters (e.g. after a change of ndte). */
int evp1d_set_params(evp1d_t *handle, const evp1d_params *params);

/* One call of the subcycle loop with host buffers: upload the fields, run
 * ndte x {stress; stepu} on the GPU, download the results.  Replaces
 * integration/ice_dyn_evp1d.F90:179-225 and src/evp_v2b.F90:91-110. */
int evp1d_run(evp1d_t *handle, int ndte, const evp1d_fields *io);

/* The same call split in three, for callers that keep the state on the GPU
 * between calls or time the device work alone. */
int evp1d_upload(evp1d_t *handle, const evp1d_fields *io);
int evp1d_subcycles(evp1d_t *handle, int ndte);
/* Subcycles that do not end a call: the same state update, without the
 * outputs the last subcycle of a call writes (strintx, strinty, Cb,
 * str1..str8).  For a caller that interleaves its own work between
 * subcycles (the velocity exchange of a split state) and ends the call with
 * evp1d_subcycles.  No counterpart in the reference. */
int evp1d_subcycles_inner(evp1d_t *handle, int n); /* device-resident */
int evp1d_download(evp1d_t *handle, const evp1d_fields *io);

/* lindividual-style loops on the device-resident state
 * (src/evp_v2b.F90:127-155): n x stress alone, n x stepu alone.  stepu_only
 * reads str1..str8 left by the last stress pass. */
int evp1d_stress_only(evp1d_t *handle, int n);
int evp1d_stepu_only(evp1d_t *handle, int n);

/* Wait for the handle's stream.  Returns EVP1D_ERR_TIMEOUT if a bounded
 * device-side wait of the solver ran out since the last check. */
int evp1d_synchronize(evp1d_t *handle);

/* Debug: a check of the timeout path; no counterpart in the reference.
 * Queues on the handle's stream one wait of the solver's own bounded kind on
 * a barrier that nothing completes, limited to `ns` nanoseconds (1e6 to 1e9).
 * It runs out and leaves its code in the handle's error word, so the next
 * evp1d_synchronize (or call that checks the word) returns EVP1D_ERR_TIMEOUT
 * and clears it; the handle stays usable. */
int evp1d_debug_wait_timeout(evp1d_t *handle, long long ns);

/* Debug: the same for the other bounded wait of the solver.  With
 * EVP1D_PERSIST=1 a call's subcycles run in one launch whose CTAs stay
 * resident (by default each subcycle is a launch of its own); before a tile loads
 * the next subcycle's state, its CTA waits on per-tile counters until the
 * tiles it depends on have finished the subcycle before.  This queues one
 * such wait on a counter that nothing raises, limited to `ns` nanoseconds
 * (1e6 to 1e9); it runs out, and the next check returns EVP1D_ERR_TIMEOUT
 * naming it.  No counterpart in the reference. */
int evp1d_debug_dep_wait_timeout(evp1d_t *handle, long long ns);

/* Debug: host-side injection of an out-of-memory failure.  The n-th device
 * allocation of the library after this call (1 = the next one) fails as if
 * the device were full: it allocates nothing, and the call that made it
 * returns EVP1D_ERR_NOMEM after freeing what it had allocated.  0 disarms.
 * Process-wide.  The reference stops the program on a failed allocation
 * instead (integration/ice_dyn_evp1d.F90:394-460). */
int evp1d_debug_fail_alloc(int n);

/* Debug: timing trace of the TMA kernel's block 0 in the last launch
 * (recorded only when EVP1D_TRACE is set at evp1d_init).  Up to 256 tiles x 8
 * %globaltimer stamps (ns): [0] the producer warps issued all of the tile's
 * copies, [1] consumer 0 has the tile's stress inputs, [2] stress done (all
 * consumers), [3] the bulk-copy warp has the tile record, [4] the tile's
 * stress slot is free, [5] consumer warp 0 finished stepu, [6] bulk copies
 * issued, [7] halo gathers issued. */
int evp1d_debug_trace(evp1d_t *handle, long long *out, int n);

/* Name of the subcycle kernel the handle runs: "fused-tile-tma" (default,
 * TMA-fed persistent kernel) or "fused-tile" (plain loads; selected by the
 * environment variable EVP1D_PATH=fused at evp1d_init). */
const char *evp1d_kernel_path(evp1d_t *handle);

/* The handle's CUDA stream (a cudaStream_t), for event timing by callers. */
void *evp1d_stream(evp1d_t *handle);

/* Number of kernel launches issued on the handle's stream since the last
 * reset (pass reset != 0 to zero the counter). */
long long evp1d_launch_count(evp1d_t *handle, int reset);

/* Message of the last error on this host thread ("" if none). */
const char *evp1d_last_error(void);

/* Library version string; it names the GPU target the library was compiled
 * for ("sm_100a"). */
const char *evp1d_version(void);

/* The compute capability the subcycle kernel's code was compiled for, as the
 * CUDA runtime reports it for `device` (major*10 + minor, 100 for sm_100a),
 * or a negative EVP1D_ERR_* code. */
int evp1d_binary_version(int device);

/* Page-locked (pinned) host memory for the arrays of evp1d_fields and
 * evp1d_grads.  Copies from and to it run at full host-link speed and are
 * asynchronous; pageable arrays work too, at lower speed.  A caller that keeps
 * its fields in such memory across timesteps (as CICE keeps its module
 * arrays) saves most of the transfer time of evp1d_run.  No counterpart in the
 * reference. */
int evp1d_host_alloc(void **ptr, size_t bytes);
int evp1d_host_free(void *ptr);

/* ----------------------------------------------------------------------------
 * Index build on the host, no GPU needed.
 * calc_2d_indices_init + calc_navel + convert_2d_1d_init
 * (integration/ice_dyn_evp1d.F90:559-589, 743-797, 1000-1087).
 * mask: [nx*ny] column-major (i fastest), nonzero = point in the 1D list.
 * Outputs are caller-allocated: indxti, indxtj [cap_na]; indxtij [cap_navel];
 * ee..sse [cap_na] 1-based.  Returns EVP1D_ERR_INVALID_ARG when a capacity is
 * too small (*na_out / *navel_out then hold the sizes needed).
 * -------------------------------------------------------------------------- */
int evp1d_build_index(int nx, int ny, int nghost, const int32_t *mask,
                      int cap_na, int cap_navel, int *na_out, int *navel_out,
                      int32_t *indxti, int32_t *indxtj, int32_t *indxtij,
                      int32_t *ee, int32_t *ne, int32_t *se, int32_t *nw,
                      int32_t *sw, int32_t *sse);

/* ----------------------------------------------------------------------------
 * 2D adapter: dyn_evp1d_init / dyn_evp1d_run / dyn_evp1d_finalize on global
 * 2D arrays (integration/ice_dyn_evp1d.F90:65-255, 326-331).  Arrays are
 * [nx*ny] column-major (i fastest) including the ghost cells, nx = nx_global
 * + 2*nghost as the adapter's G_* arrays (:93-94).  init builds the 1D list
 * from tmask (:559-589, 743-816); run copies the 2D arrays to the GPU, where
 * kernels derive skipT/skipU from the ice masks (set_skipMe, :521-537),
 * gather the fields onto the list with halo velocities 0 (convert_2d_1d_dyn,
 * :818-882), run ndte subcycles and scatter the results back
 * (convert_1d_2d_dyn, :884-947); the arrays come back whole, so cells outside
 * the list keep the caller's values.  Unlike the reference, whose L_*
 * arguments are intent(in), results are returned in the inout arrays.  With
 * the arrays in evp1d_host_alloc memory the copies run at full speed.
 * -------------------------------------------------------------------------- */
typedef struct evp1d_dyn_fields {
  double *stress[12];          /* inout: stressp_1..4, stressm_1..4, stress12_1..4 */
  const double *strength;      /* in */
  const double *cdn_ocn, *aiu, *uocn, *vocn, *waterxU, *wateryU;  /* in */
  const double *forcexU, *forceyU, *umassdti, *fmU, *Tbu;          /* in */
  double *strintxU, *strintyU, *Cb;  /* inout: written at ice U points */
  double *uvel, *vvel;               /* inout */
  const int32_t *icetmask, *iceumask;  /* in, nonzero = ice */
} evp1d_dyn_fields;

typedef struct evp1d_dyn_handle evp1d_dyn_t;

int evp1d_dyn_init(evp1d_dyn_t **handle, int nx, int ny, int nghost,
                   const int32_t *tmask, const double *dyT, const double *dxT,
                   const double *uarear, const double *HTE, const double *HTN,
                   const evp1d_params *params, int device);
int evp1d_dyn_run(evp1d_dyn_t *handle, int ndte, const evp1d_dyn_fields *io);
int evp1d_dyn_finalize(evp1d_dyn_t *handle);
/* Number of 1D list points (nActive) and slots (navel) of a 2D handle. */
int evp1d_dyn_sizes(evp1d_dyn_t *handle, int *na, int *navel);

/* Largest tile compute set (owned points plus recomputed forward-halo
 * points; one kernel thread each) of the tile plans of handles created after
 * the call (evp1d_init, evp1d_init_batched, and evp1d_plan_stats); 32..256,
 * default 256.  Process-wide; handles that exist keep their plan.  No
 * counterpart in the reference: a dimension for the autotuner
 * (evp1d.tune_tile_points in the Python binding times candidate sizes on the
 * caller's problem).  Results do not depend on it. */
int evp1d_set_tile_points(int points);
int evp1d_get_tile_points(void);

/* ----------------------------------------------------------------------------
 * Velocity exchange of one state split over several handles (one per GPU).
 * No counterpart in the reference, which gathers the whole domain onto the
 * master task before the 1D solver runs (gather_global_ext,
 * integration/ice_dyn_evp1d.F90:637-716).
 *
 * Each handle holds a band of the global list plus ghost points: the stepu
 * neighbours of its band (solved for stress here, skipU set) and the other
 * points whose velocities its stress reads (halo slots).  After every
 * subcycle, the caller gathers the band's boundary velocities, moves them to
 * the handles that hold them as ghosts, and scatters them there.
 *   evp1d_exchange_setup:  send_idx are the 1-based local list points
 *                          (1..na) whose u, v the handle sends; recv_idx are
 *                          the 1-based local positions (1..navel, no repeats)
 *                          that receive u, v.
 *                          It also allocates a send and a receive buffer
 *                          on the device (evp1d_exchange_buffers).
 *   evp1d_exchange_pack:   device buffer[2k], [2k+1] = u, v of send_idx[k] in
 *                          the current state (2 x n_send doubles); a NULL
 *                          buffer means the handle's send buffer.
 *   evp1d_exchange_unpack: u, v of recv_idx[k] in the current state =
 *                          device buffer[2k], [2k+1] (2 x n_recv doubles); a
 *                          NULL buffer means the handle's receive buffer.
 *   evp1d_exchange_buffers: device addresses of the handle's send and
 *                          receive buffers (NULL when empty), valid until the
 *                          next setup or finalize: what CUDA-aware MPI or
 *                          NCCL sends from and receives into.
 * Pack and unpack run on the handle's stream (evp1d_stream) and do not wait
 * for it.  Single-state handles only (not evp1d_init_batched). */
int evp1d_exchange_setup(evp1d_t *handle, int n_send, const int32_t *send_idx, int n_recv,
                         const int32_t *recv_idx);
int evp1d_exchange_pack(evp1d_t *handle, double *dev_buffer);
int evp1d_exchange_unpack(evp1d_t *handle, const double *dev_buffer);
int evp1d_exchange_buffers(evp1d_t *handle, double **send, double **recv);

/* ----------------------------------------------------------------------------
 * Host-only diagnostics of the tile plan the solver would build for a 1D
 * problem (same arguments as evp1d_init, 1-based neighbours; no GPU needed).
 * stats[0] tiles, [1] device slots (list points + alignment padding),
 * [2] forward-halo points summed over tiles, [3] 1 if the tiles follow grid
 * coordinates rebuilt from the neighbour vectors (0: consecutive list points),
 * [4] largest halo of one tile, [5] largest tile, [6] largest number of
 * extra velocity points (read by the stencil, owned by no tile point) of one
 * tile, [7] largest number of tiles in one run (the tiles one CTA of the
 * subcycle kernel works through; the plan is made for 148 CTAs, a B200's SM
 * count).
 * -------------------------------------------------------------------------- */
int evp1d_plan_stats(int na, int navel, const int32_t *ee, const int32_t *ne,
                     const int32_t *se, const int32_t *nw, const int32_t *sw,
                     const int32_t *sse, long long stats[8]);
/* Builds the same plan and decodes every index the kernels gather through
 * (slot maps, tile ranges, neighbour slots, forward halos, extra velocity
 * points, the packed local indices), comparing each with what the neighbour
 * vectors say it must be.  EVP1D_OK, or EVP1D_ERR_INDEX naming the first
 * violation; *violations (may be NULL) gets their number.  Host only.  With
 * the environment variable EVP1D_CHECK_PLAN set, evp1d_init and
 * evp1d_init_batched run the same check and refuse a plan that fails it. */
int evp1d_plan_check(int na, int navel, const int32_t *ee, const int32_t *ne,
                     const int32_t *se, const int32_t *nw, const int32_t *sw,
                     const int32_t *sse, long long *violations);

/* ----------------------------------------------------------------------------
 * Adjoint (reverse-mode gradients) of the subcycle loop.  No counterpart in
 * the reference, whose loop is forward only.
 *
 * 1. evp1d_run_checkpointed: the same call as evp1d_run, recording what the
 *    reverse sweep needs on the device:
 *      interval > 0:  (u, v, 12 stresses) at the start of every
 *                     `interval` subcycles, except that the velocities of
 *                     the last segment are taped; the sweep recomputes each
 *                     checkpointed segment's velocities from its checkpoint
 *                     (one extra forward, less the last segment);
 *      interval <= 0: sized to device memory (the budget of
 *                     evp1d_set_adjoint_budget, default 80% of the free
 *                     memory): every subcycle's velocities when they fit (no
 *                     recompute); else checkpoints at the interval
 *                     ceil(sqrt(ndte * checkpoint size / velocity size)) for
 *                     the first subcycles and every velocity state for as
 *                     many final subcycles as the budget holds, so only the
 *                     checkpointed head is recomputed.
 * 2. evp1d_adjoint: given dJ/d uvel, dJ/d vvel of the call's final list-point
 *    velocities ([na], host) and optionally dJ/d of the final stresses
 *    (lam_stress: NULL, or 12 pointers of which any may be NULL), writes the
 *    requested gradients ([na] host arrays; NULL = not wanted):
 *      strength, Cw (per point; for a scalar Cw sum them), forcex, forcey,
 *      uvel, vvel, stress[12] (with respect to the call's starting values),
 *      uvel_init, vvel_init (only when the recorded call passed them; when
 *      it did not, their gradient is part of uvel, vvel and these are 0).
 * Derivatives take the branch the forward took at max(Delta, DminArea) and
 * are 0 at a zero-length square root.  They are computed in FP64 with fused
 * multiply-adds (they are not bit-matched to anything; the values that pick
 * a branch are recomputed with the forward's own rounding), so the same
 * recording and seed give the same bits on every sweep, and a batched member
 * the bits of the member solved alone.  The recorded forward is dropped by the
 * next evp1d_upload or evp1d_set_params; one recording can be swept any
 * number of times with different seeds.  Works on batched handles (gradients
 * per member in the member-major [na] layout).
 * -------------------------------------------------------------------------- */
typedef struct evp1d_grads {
  double *strength, *Cw, *forcex, *forcey;
  double *uvel, *vvel;
  double *stress[12];
  double *uvel_init, *vvel_init;
} evp1d_grads;

int evp1d_run_checkpointed(evp1d_t *handle, int ndte, const evp1d_fields *io,
                           int interval);
int evp1d_adjoint(evp1d_t *handle, const double *lam_uvel, const double *lam_vvel,
                  const double *const *lam_stress, const evp1d_grads *grads);
/* The same two calls split for device-resident timing: the recording forward
 * after evp1d_upload; the seed upload, the reverse sweep (queued on the
 * handle's stream) and the gradient download. */
int evp1d_record_subcycles(evp1d_t *handle, int ndte, int interval);
int evp1d_adjoint_seed(evp1d_t *handle, const double *lam_uvel, const double *lam_vvel,
                       const double *const *lam_stress);
int evp1d_adjoint_sweep(evp1d_t *handle);
int evp1d_adjoint_gradients(evp1d_t *handle, const evp1d_grads *grads);
/* Device memory for checkpoints and tape of later sized recordings
 * (interval <= 0); 0 restores the default, 80% of the free memory.  A
 * budget below what checkpointing at the memory-minimising interval needs
 * gets that minimum. */
int evp1d_set_adjoint_budget(evp1d_t *handle, long long bytes);
/* info[0] 1 if a recorded forward is held, [1] subcycles on the velocity
 * tape (the final ones), [2] checkpoint interval, [3] checkpoints, [4] bytes
 * of checkpoints and tape, [5] bytes of the adjoint work arrays, [6] bytes of
 * the forward solver, [7] kernel launches of the last sweep. */
int evp1d_adjoint_info(evp1d_t *handle, long long info[8]);

/* ----------------------------------------------------------------------------
 * Allocation-free entry point.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory -- device memory owned by
 * another runtime or memory pool, or code where a cudaMalloc would
 * synchronise the device or fail -- and that already hold the 1D problem in
 * device memory.  One call runs ndte x {stress; stepu} in place on the
 * caller's device arrays in the reference 1D layout, exactly as evp1d_run
 * does on host arrays, with the reference-order stress and stepu kernels.
 *
 * - Every pointer (neighbours, geometry, every field of `io`) is device (or
 *   managed) memory of the calling thread's current device; neighbours are
 *   1-based as in evp1d_init; skipT/skipU nonzero = skip.  uvel_init/
 *   vvel_init may both be NULL (= the velocities at call start); str[k] may be
 *   NULL (str1..str8 are then not returned).
 * - The call allocates nothing.  str1..str8 and the call-start velocities
 *   live in one fixed device array of the library holding navel up to
 *   EVP1D_NOALLOC_MAX_NAVEL (10 arrays of that many doubles, 20 MiB);
 *   a larger navel is rejected with EVP1D_ERR_INVALID_ARG.
 * - str1..str8 are cleared at the start of every call.  Every call on a
 *   device shares that array, so calls that overlap on the GPU (from several
 *   host threads, or on streams that run concurrently) race; serialise them.
 * - Every call looks up the array's device address in the current context
 *   (a lookup that allocates nothing), so a cudaDeviceReset or a context of
 *   the caller's own between calls is safe.
 * - Work is queued on `stream` (a cudaStream_t; NULL = the legacy default
 *   stream) and the call returns after the stream has finished it (it reads
 *   the index check back).
 *   Neighbours outside 1..navel give EVP1D_ERR_INDEX before any array is
 *   written.
 * -------------------------------------------------------------------------- */
#define EVP1D_NOALLOC_MAX_NAVEL 262144
int evp1d_run_device_noalloc(int na, int navel, const int32_t *ee,
                             const int32_t *ne, const int32_t *se,
                             const int32_t *nw, const int32_t *sw,
                             const int32_t *sse, const double *dxT,
                             const double *dyT, const double *HTE,
                             const double *HTN, const double *HTEm1,
                             const double *HTNm1, const double *uarear,
                             const evp1d_params *params, int ndte,
                             const evp1d_fields *io, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* EVP1D_H */
