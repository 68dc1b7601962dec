/*
 * susy_b200.h -- C ABI of the B200 implementation of the 4d_Q16 RHMC
 * fermion path of SUSY LATTICE (daschaich/susy).
 *
 * Every entry point is plain C: opaque handle, plain pointers and sizes, no
 * CUDA or torch types.  Host arrays use the reference's own memory layout
 * so a reference build can hand its arrays over unchanged:
 *   - sites in node_index order (4d_Q16/generic/layout_hyper_prime.c:157),
 *   - a matrix is e[NCOL][NCOL] of {double real, imag} (include/susy.h:28),
 *   - a Twist_Fermion is {Fsite, Flink[5], Fplaq[10]} (susy/lattice.h:18),
 *   - link-type fields (links, momenta) are 5 matrices per site, read with a
 *     caller-given byte stride between sites, so &lattice[0].link[0] with
 *     stride sizeof(site) (susy/lattice.h:29-59) works without a copy.
 * Lattice fields live on the GPU between calls (links, momenta, derived
 * fields); Twist_Fermion arguments are copied in and out per call.
 *
 * Return values: entry points return SUSY_B200_OK (0) or a negative error
 * code unless documented otherwise; susy_b200_last_error() keeps the first
 * error.  Nothing here terminates the process or waits without bound.
 * One handle must not be used from two host threads at once (the reference
 * is single threaded per rank, susy/lattice.h globals).
 */
#ifndef SUSY_B200_H
#define SUSY_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SUSY_B200_OK 0
#define SUSY_B200_EINVAL -1      /* bad argument (e.g. sign not +-1)    */
#define SUSY_B200_ECUDA -2       /* CUDA runtime error                   */
#define SUSY_B200_ENOMEM -3      /* device allocation failed             */
#define SUSY_B200_ENOCONV -4     /* solver hit its iteration limit       */
#define SUSY_B200_ENAN -5        /* non-finite value detected            */
#define SUSY_B200_ESCRATCH -6    /* field larger than the fixed scratch of
                                    susy_b200_DSq_noalloc                 */

typedef struct susy_b200_lattice susy_b200_lattice;

/* Lattice geometry and action couplings: the reference globals the hot
 * path reads (susy/lattice.h:76-100, set in susy/setup.c:307-557). */
typedef struct {
  int nx, ny, nz, nt;      /* lattice.h:76                                  */
  int ncol;                /* NCOL, include/susy.h:16; 2, 3 or 4            */
  int pbc;                 /* PBC, lattice.h:78; +1 or -1 temporal fermion BC */
  double kappa;            /* NCOL / (4 lambda), setup.c:459                 */
  double bmass;            /* scalar potential coupling, lattice.h:98        */
  double fmass;            /* fermion mass, DSq adds fmass^2 (utilities.c:880) */
  double kappa_u1;         /* plaquette determinant action, action.c:212     */
  double G;                /* determinant coupling; doG = G > 1e-8 (setup.c:450) */
  int iseed;               /* seeds the per-site generators (make_lattice.c:48) */
  int device;              /* CUDA device ordinal                            */
} susy_b200_params;

/* ---- lifetime ---------------------------------------------------------- */
/* Replaces the field allocation of setup() / make_fields()
 * (susy/setup.c:126-260).  Returns NULL on failure. */
susy_b200_lattice *susy_b200_create(const susy_b200_params *p);
void susy_b200_destroy(susy_b200_lattice *h);
int susy_b200_last_error(const susy_b200_lattice *h);
const char *susy_b200_error_string(int code);
/* Launch on this cudaStream_t (passed as void*); NULL = the handle's own. */
int susy_b200_set_stream(susy_b200_lattice *h, void *cuda_stream);
/* The cudaStream_t (as void*) the handle launches on: its own non-blocking
 * stream unless susy_b200_set_stream chose another; NULL for a NULL handle. */
void *susy_b200_get_stream(const susy_b200_lattice *h);
int susy_b200_sync(susy_b200_lattice *h);
int susy_b200_volume(const susy_b200_lattice *h);
/* Number of kernels this library has launched in this process (all handles);
 * no reference counterpart, used to account GPU work in benchmarks. */
long long susy_b200_launch_count(void);

/* ---- gauge field and momenta (site.link / site.mom, lattice.h:37-45) --- */
/* Upload links and recompute every derived field, as readin() and
 * update_u() leave them (setup.c:551-554, update_o.c:31-34). */
int susy_b200_set_links(susy_b200_lattice *h, const double *links, size_t site_stride_bytes);
int susy_b200_get_links(susy_b200_lattice *h, double *links, size_t site_stride_bytes);
int susy_b200_set_mom(susy_b200_lattice *h, const double *mom, size_t site_stride_bytes);
int susy_b200_get_mom(susy_b200_lattice *h, double *mom, size_t site_stride_bytes);

/* ---- derived fields ---------------------------------------------------- */
/* compute_plaqdet()  susy/utilities.c:17   (also ZW* = plaqdet (plaqdet-1)^*) */
int susy_b200_compute_plaqdet(susy_b200_lattice *h);
/* compute_Uinv()     susy/utilities.c:117 */
int susy_b200_compute_Uinv(susy_b200_lattice *h);
/* compute_DmuUmu()   susy/action.c:15 */
int susy_b200_compute_DmuUmu(susy_b200_lattice *h);
/* compute_Fmunu()    susy/action.c:71 */
int susy_b200_compute_Fmunu(susy_b200_lattice *h);
/* Copy out derived fields: plaqdet as [V][5][5] complex (diagonal zero),
 * DmuUmu as [V] matrices, Fmunu as [V][10], Uinv as [V][5]; node_index order. */
int susy_b200_get_derived(susy_b200_lattice *h, double *plaqdet, double *DmuUmu,
                          double *Fmunu, double *Uinv);

/* ---- fermion operator -------------------------------------------------- */
/* void fermion_op(Twist_Fermion *src, Twist_Fermion *dest, int sign)
 *   susy/utilities.c:765; sign must be +1 (D) or -1 (D^dag), otherwise
 *   SUSY_B200_EINVAL (the reference calls terminate(1), utilities.c:789). */
int susy_b200_fermion_op(susy_b200_lattice *h, const double *src, double *dest, int sign);
/* void DSq(Twist_Fermion *src, Twist_Fermion *dest)   susy/utilities.c:874 */
int susy_b200_DSq(susy_b200_lattice *h, const double *src, double *dest);

/* ---- multi-shift CG ------------------------------------------------------ */
/* int congrad_multi(Twist_Fermion *src, Twist_Fermion **psim, int MaxCG,
 *                   Real errormin, Real *size_r)   susy/congrad_multi.c:26
 * The reference reads Norder and shift[] from globals; here they are
 * arguments.  Returns the iteration count (>= 0) or a negative error code;
 * *size_r receives the final |r|^2.  Reaching MaxCG is not an error, as in
 * the reference (congrad_multi.c:182). */
int susy_b200_congrad_multi(susy_b200_lattice *h, const double *src, double *const *psim,
                            int norder, const double *shift, int MaxCG, double errormin,
                            double *size_r);

/* ---- device-resident fields (no host copies) --------------------------- */
/* A Twist_Fermion in device layout; prec is 64 (FP64) or 32 (FP32). */
void *susy_b200_tf_alloc(susy_b200_lattice *h, int prec);
void susy_b200_tf_free(susy_b200_lattice *h, void *dev);
size_t susy_b200_tf_bytes(const susy_b200_lattice *h, int prec);
int susy_b200_tf_upload(susy_b200_lattice *h, void *dev, int prec, const double *host_tf);
int susy_b200_tf_download(susy_b200_lattice *h, const void *dev, int prec, double *host_tf);
int susy_b200_tf_convert(susy_b200_lattice *h, const void *src, int prec_src, void *dst,
                         int prec_dst);
int susy_b200_dev_fermion_op(susy_b200_lattice *h, const void *src, void *dst, int sign,
                             int prec);
/* Operator kernel selection (no reference counterpart: the reference has one
 * CPU loop nest).  autotune times every variant on this lattice and keeps
 * the fastest per precision; it also runs by itself on first use.
 * fop_variant returns the current variant of a precision, sets it when
 * set_to >= 0 and copies the autotuner's ms per variant when ms != NULL. */
/* Per-trajectory measurements printed by control.c:85-138, on the
 * handle's current links (and the derived fields of the last link update).
 * Field by field the reference function and output line it reproduces. */
typedef struct {
  double linktr[5], linktr_ave, linktr_width;   /* link_trace.c:9, FLINK      */
  double link_det[5], det_ave, det_width;       /* link_trace.c:9, FLINK_DET  */
  double ploop_re, ploop_im, ploop_mod;         /* ploop(TUP, NODET), GMES    */
  double ss_plaq, st_plaq;                      /* plaquette, plaq.c:7, GMES  */
  double gauge_action;                          /* gauge_action(NODET),
                                                   action.c:106; BACTION is
                                                   this / volume             */
  double lines_re[5], lines_im[5];              /* ploop(dir, NODET), LINES   */
  double lines_polar_re[5], lines_polar_im[5];  /* ploop(dir, YESDET),
                                                   LINES_POLAR                */
  double det_tot_re, det_tot_im, det_sq_re, det_sq_im, det_wsq;
                                                /* measure_det,
                                                   determinant.c:92, DET      */
  double width_plaq, width_det_re, width_det_im; /* widths.c:8, WIDTHS        */
  double uubar_ave[4], uubar_width[4], uubar_min[4], uubar_max[4];
                                                /* scalar_eig(NODET),
                                                   scalar_eig.c:15, UUBAR_EIG */
  double polar_ave[4], polar_width[4], polar_min[4], polar_max[4];
                                                /* scalar_eig(YESDET),
                                                   POLAR_EIG (first NCOL used) */
} susy_b200_meas;
int susy_b200_measure(susy_b200_lattice *h, susy_b200_meas *m);
/* plaquette(double *ss_plaq, double *st_plaq), plaq.c:7 */
int susy_b200_plaquette(susy_b200_lattice *h, double *ss_plaq, double *st_plaq);

/* FP64 multi-shift CG vector update (no reference counterpart; the
 * reference's congrad_multi.c:109-150 updates psi_j and p_j of every live
 * shift every iteration).  on = 1 (default): one pass per 8 iterations
 * advances every psi_j and p_j with the combined coefficients of those
 * iterations (same recurrences and stopping rules, summed in a different
 * order); on = 0: the per-iteration update.  on < 0 only queries.
 * Returns the previous setting. */
int susy_b200_cg_blocked(susy_b200_lattice *h, int on);
/* Iterations each shift of the last multi-shift solve on this handle took
 * (no reference counterpart; congrad_multi.c:154-165 freezes shift j once
 * zeta_j^2 |r|^2 <= rsqstop and updates it no more): iters[j] = the
 * iteration at which shift j froze, the solve's iteration count for the
 * base shift and for shifts that never froze.  1 <= norder <= 32. */
int susy_b200_cg_freeze_iterations(susy_b200_lattice *h, int *iters, int norder);
/* Solver launch mode (no reference counterpart): on = 1 (default) captures
 * the ~100 kernel launches of 16 solver iterations into a CUDA graph once
 * per solve and operator precision and replays it; on = 0 launches them
 * one by one.  Same kernels, same results.  on < 0 only queries; returns
 * the previous setting. */
int susy_b200_use_graphs(susy_b200_lattice *h, int on);
/* Trajectory pseudofermion solves (no reference counterpart; the reference
 * solves them one after the other, update_o.c:98-113): on = 1 (default)
 * with Nroot >= 2 the odd pseudofermions' solves run on a second solver
 * context of the handle (its own stream and scratch, about as much device
 * memory again as one solve's fields; made on first use) from a second host
 * thread while the calling thread runs the even ones, so the solves overlap
 * on the GPU; on = 0 solves them in turn on the handle's stream.  Same
 * kernels on the same data: the same results.  on < 0 only queries;
 * returns the previous setting. */
int susy_b200_pf_streams(susy_b200_lattice *h, int on);
/* Solver behind susy_b200_congrad_multi (the host-array drop-in for
 * congrad_multi.c:26): SUSY_B200_SOLVER_FP64 (default, the reference's
 * recurrences) or SUSY_B200_SOLVER_MIXED (same FP64 true-residual bound).
 * Returns the previous setting. */
int susy_b200_set_solver(susy_b200_lattice *h, int solver);
/* Mixed-precision solver settings (no reference counterpart): the operator
 * runs in FP32 once |r| < fp32_below |src| (default 3e-4; fp32_below = 1
 * runs it in FP32 from the first iteration); with the FP32 operator the
 * FP64 true residual replaces the iterated one whenever |r| fell by
 * reliable_factor (default 1e-2) since the last replacement.
 * 0 < fp32_below <= 1, 0 < reliable_factor < 1, else SUSY_B200_EINVAL. */
int susy_b200_mixed_params(susy_b200_lattice *h, double fp32_below, double reliable_factor);
/* Mixed solver: iters > 0 replaces the reliable_factor trigger by a fixed
 * schedule, the FP64 true residual at the first 8-iteration block boundary
 * at least iters iterations after the previous replacement (or after the
 * switch to FP32); 0 (default) restores the residual trigger.  iters < 0:
 * SUSY_B200_EINVAL. */
int susy_b200_mixed_reliable_interval(susy_b200_lattice *h, int iters);
/* Mixed solver, after the multi-shift pass: a shift whose FP64 true
 * residual is above the bound gets correction solves (D^dag D + sigma) e = r,
 * x += e, with the FP32 operator and recurrences (fp32 = 1, the default;
 * the FP64 true residual is checked after every pass) or in FP64 (fp32 = 0).
 * No counterpart in the reference.  fp32 not 0 or 1: SUSY_B200_EINVAL. */
int susy_b200_mixed_correction(susy_b200_lattice *h, int fp32);
/* The reference's compile-time RESCALE option (susy/defines.h:30; its
 * susy_cheb and susy_mode targets define it): fermion_op doubles the site
 * component of its input and of its output (utilities.c:795-797,841-844),
 * for every operator application of the handle (fermion_op, DSq and the
 * solvers; the fermion force, which the reference marks "not yet
 * conserving" under RESCALE, update_h.c:697-702, is unchanged).  on = 1
 * sets it, 0 clears it, < 0 only queries; returns the previous setting. */
int susy_b200_set_rescale(susy_b200_lattice *h, int on);
/* Mixed solver, its FP32-operator phase: the residual ring and the
 * operator's input held in FP32 (fp32 = 1; the shifted search vectors, the
 * solutions, the recurrences and every residual replacement stay FP64) or
 * in FP64 (fp32 = 0, the default: on the 12^3x24 U(3) benchmark the FP32
 * residuals cost more correction iterations than they save).  No
 * counterpart in the reference.
 * fp32 < 0 only queries; returns the previous setting. */
int susy_b200_mixed_vectors(susy_b200_lattice *h, int fp32);
#define SUSY_B200_FOP_NVARIANTS 15   /* entries of ms_per_variant */
int susy_b200_autotune(susy_b200_lattice *h);
int susy_b200_fop_variant(susy_b200_lattice *h, int prec, int set_to, float *ms_per_variant);
int susy_b200_dev_DSq(susy_b200_lattice *h, const void *src, void *dst, int prec);
/* dst = (D^dag D + fmass^2) src without allocating any device memory.
 * No counterpart in the reference.  For callers that own every device
 * buffer themselves and must not have a library call cudaMalloc (an
 * application with its own device memory pool, or code that cannot afford
 * the device-wide synchronisation an allocation may cause): no handle is
 * needed and the library calls no allocation routine.  All
 * pointers are FP64 device fields in the device layout (structure of
 * arrays, lexicographic sites x + nx (y + ny (z + nz t)), site stride
 * S = volume rounded up to a multiple of 32, complex {re, im} doubles):
 *   links [5][ncol][ncol][S], src and dst [16][ncol][ncol][S];
 *   Uinv [5][ncol][ncol][S] (inverse links) and plaqdet [25][S]
 *   (plaquette determinants [a][b], as compute_plaqdet forms them) are read
 *   only when G > 1e-8 and may be NULL otherwise.
 * The intermediate field D src lives in one fixed 16 MiB device array inside
 * the library (2^20 complex doubles, so 16 ncol^2 S <= 2^20, e.g. 8^4 sites
 * for any ncol); larger lattices return SUSY_B200_ESCRATCH.  Every call on
 * a device shares that array: calls whose kernels overlap on the GPU (other
 * streams, other host threads) race and must be serialised by the caller.
 * The library's modules load lazily: the first call on each device loads
 * this one, and the driver reserves the 16 MiB array at that moment (with
 * whatever synchronisation a module load implies).  Make that first call at
 * set-up time, before any stream capture.  Every call looks the array's
 * device address up again, so a cudaDeviceReset in between is harmless.
 * Extents must be even and >= 2 and ncol 2..4 (else SUSY_B200_EINVAL);
 * the volume is formed in 64 bits, so extents whose product would wrap a
 * 32-bit int return SUSY_B200_ESCRATCH.  Launches on cuda_stream
 * (NULL = default stream) and returns without synchronising. */
int susy_b200_DSq_noalloc(int nx, int ny, int nz, int nt, int ncol, int pbc, double G,
                          double fmass, const void *links, const void *Uinv,
                          const void *plaqdet, const void *src, void *dst, void *cuda_stream);
int susy_b200_dev_congrad_multi(susy_b200_lattice *h, const void *src, void *const *psim,
                                int norder, const double *shift, int MaxCG, double errormin,
                                double *size_r, int *iters);
/* Same solve with the mixed-precision solver (FP32 multi-shift pass, then
 * FP64 true-residual defect correction per shift): every shift ends with
 * |src - (D^dag D + shift_j) psim_j|^2 <= errormin |src|^2 in FP64, unless
 * MaxCG operator applications run out.  *size_r = worst final true |r|^2;
 * *iters = operator applications (multi-shift pass plus refinement). */
int susy_b200_dev_congrad_multi_mixed(susy_b200_lattice *h, const void *src, void *const *psim,
                                      int norder, const double *shift, int MaxCG,
                                      double errormin, double *size_r, int *iters);

/* ---- forces, link update, actions ------------------------------------- */
/* double gauge_force(Real eps)   susy/update_h.c:15 (includes det_force
 * when kappa_u1 > 0, update_h.c:257); mom -= kappa eps f_U^dag;
 * *norm = eps sqrt(sum |f|^2) / volume as the reference returns. */
int susy_b200_gauge_force(susy_b200_lattice *h, double eps, double *norm);
/* double det_force(Real eps)     susy/det_force.c:6; *norm = sum |f|^2 */
int susy_b200_det_force(susy_b200_lattice *h, double eps, double *norm);
/* double fermion_force(Real eps, Twist_Fermion *src, Twist_Fermion **sol)
 *   susy/update_h.c:928; Norder and amp4[] (globals there) are arguments.
 *   src is accepted and ignored, as in the reference. */
int susy_b200_fermion_force(susy_b200_lattice *h, double eps, const double *src,
                            const double *const *sol, int norder, const double *amp4,
                            double *norm);
int susy_b200_dev_fermion_force(susy_b200_lattice *h, double eps, void *const *sol, int norder,
                                const double *amp4, double *norm);
/* void update_u(Real eps)  susy/update_o.c:20: link += eps mom, then the
 * derived fields are recomputed. */
int susy_b200_update_u(susy_b200_lattice *h, double eps);
/* double action(src, sol)  susy/action.c:293.  parts receives
 * {gauge, bmass, det, fermion (summed over roots), mom}; sol holds
 * nroot * norder arrays, root-major. */
int susy_b200_action(susy_b200_lattice *h, int nroot, const double *const *src,
                     const double *const *sol, int norder, const double *amp4, double ampdeg4,
                     double *parts);

/* ---- random fields (per-site generators, generic/ranstuff.c) ----------- */
/* (Re)seed every site generator and the node generator as setup() does
 * (make_lattice.c:48, setup.c:246); create() already seeds with p->iseed. */
int susy_b200_seed(susy_b200_lattice *h, int iseed);
/* void ranmom()   susy/grsource.c:44: fills the device momenta */
int susy_b200_ranmom(susy_b200_lattice *h);
/* Gaussian Twist_Fermion R in grsource's draw order (grsource.c:213-245) */
int susy_b200_gaussian_tf(susy_b200_lattice *h, double *out);

/* ---- RHMC trajectory ---------------------------------------------------- */
#define SUSY_B200_SOLVER_FP64 0    /* congrad_multi as the reference runs it   */
#define SUSY_B200_SOLVER_MIXED 1   /* FP32 multi-shift + FP64 residual refinement */
#define SUSY_B200_MAX_NROOT 4
#define SUSY_B200_HMC 0            /* update_o.c:127 as built for susy_hmc      */
#define SUSY_B200_SMD 1            /* the same with SMD_ALGORITHM (susy_smd)    */

/* Rational approximation and integrator parameters: the reference globals
 * of susy/lattice.h:116-124 and setup_rhmc.c (amp4/shift4/amp8/shift8/
 * ampdeg4/ampdeg8 for Norder poles), nsteps[2], traj_length, niter and
 * rsqmin = error_per_site^2 (setup.c:356-359). */
typedef struct {
  int Nroot, Norder;
  const double *amp4, *shift4, *amp8, *shift8;
  double ampdeg4, ampdeg8;
  int nsteps[2];
  double traj_length;
  int niter;
  double rsqmin;
  int solver;          /* SUSY_B200_SOLVER_FP64 or SUSY_B200_SOLVER_MIXED */
  int no_metropolis;   /* 1: keep the end of every trajectory and only report
                          delta S, as the reference's non-HMC build does
                          (update_o.c:252-255) */
  int algorithm;       /* SUSY_B200_HMC (0) or SUSY_B200_SMD */
  double friction;     /* SMD friction (lattice.h:79, read at setup.c:324):
                          momenta refreshed as mom <- c1 mom + c2 gaussian,
                          c1 = exp(-traj_length friction) (0 if friction < 0),
                          c1^2 + c2^2 = 1 (grsource.c:13-40); pseudofermion
                          sources src <- c2 (fresh source) + c1 src with the
                          reference's integer c1, c2 (grsource.c:74-197): a
                          fresh source unless friction == 0, which keeps the
                          previous trajectory's source */
} susy_b200_rhmc;

/* What update() prints (update_o.c:244-277) */
typedef struct {
  double delta_S, start_S, end_S, xrandom;
  double start_parts[5], end_parts[5];   /* gauge, bmass, det, fermion, mom */
  int accept, iters;
  double gnorm, max_gf;
  double fnorm[SUSY_B200_MAX_NROOT], max_ff[SUSY_B200_MAX_NROOT];
} susy_b200_traj;

/* int grsource(Twist_Fermion *src)   susy/grsource.c:200; returns CG iterations */
int susy_b200_grsource(susy_b200_lattice *h, const susy_b200_rhmc *r, double *src);
/* void smdmom(Real eps)   susy/grsource.c:13 (friction passed explicitly):
 * mom <- c1 mom + c2 (gaussian momenta as ranmom draws them),
 * c1 = exp(-eps friction), 0 when friction < 0, c2 = sqrt(1 - c1^2) */
int susy_b200_smdmom(susy_b200_lattice *h, double eps, double friction);
/* int update()   susy/update_o.c:127: one HMC trajectory (momentum refresh,
 * pseudofermions, Omelyan integration, Metropolis with the node generator).
 * Returns the CG iteration count or a negative error code. */
int susy_b200_update(susy_b200_lattice *h, const susy_b200_rhmc *r, susy_b200_traj *res);
/* update() with the refreshed momenta and pseudofermion sources replaced by
 * the given ones (mom: link-type array; src: Nroot Twist_Fermion arrays),
 * to replay a trajectory from known fields. */
int susy_b200_update_replay(susy_b200_lattice *h, const susy_b200_rhmc *r, susy_b200_traj *res,
                            const double *mom, const double *const *src);

/* ---- Learned preconditioner (no reference counterpart) ------------------
 * A gauge-covariant network bound to a lattice handle (it reads the
 * handle's current links): Twist_Fermion -> 16 site-type channels (each
 * component's path closed with inverse links), three layers of
 * parallel-transported nearest-neighbour convolutions 16 -> 32 -> 32 -> 16
 * (11 taps: the site and both directions of the five links), back to a
 * Twist_Fermion.  bfloat16 weights, FP32 arithmetic, FP64 device
 * Twist_Fermions in and out.  Weights (susy_b200_net_nweights() complex
 * numbers, re/im interleaved) are layer by layer W[tap][c_out][c_in]. */
typedef struct susy_b200_net susy_b200_net;
int susy_b200_net_nweights(void);
susy_b200_net *susy_b200_net_create(susy_b200_lattice *h);
void susy_b200_net_destroy(susy_b200_net *n);
int susy_b200_net_set_weights(susy_b200_net *n, const double *w);
int susy_b200_net_apply(susy_b200_net *n, const void *src, void *dst);
/* net_apply's channel mixes: on the tensor cores (on = 1, the default; the
 * transports rounded to bfloat16, mma.sync BF16 x BF16 products with FP32
 * accumulation) or as FP32 multiply-adds (on = 0).  Training
 * (net_loss_grad*) always runs the FP32 forward pass it differentiates.
 * on < 0 only queries; returns the previous setting. */
int susy_b200_net_tensor_cores(susy_b200_net *n, int on);
/* loss = |N(r) - e|^2 / |e|^2 for device Twist_Fermions r, e; when grad is
 * not NULL, grad += dL/dW* (complex interleaved, the layout of set_weights:
 * dL/dRe w = 2 Re, dL/dIm w = 2 Im) */
int susy_b200_net_loss_grad(susy_b200_net *n, const void *r, const void *e, double *loss,
                            double *grad);
/* The same with sigma >= 0: the A-norm error (d, A d) / (e, A e), d = N(r) - e,
 * A = D^dag D + fmass^2 + sigma (e = A^-1 r, so (e, A e) = Re<e, r>);
 * sigma < 0 is the plain relative error above. */
int susy_b200_net_loss_grad2(susy_b200_net *n, const void *r, const void *e, double sigma,
                             double *loss, double *grad);

/* Multi-shift solve with learned preconditioning (config "FP32+learned"):
 * the FP64 multi-shift stops the smallest (base) shift at loose |src|^2
 * while the others freeze at errormin |src|^2 as usual; every shift whose
 * FP64 true residual is still above errormin |src|^2 is then refined by
 * flexible CG, preconditioned by net for the nrefine smallest shifts (net
 * NULL: unpreconditioned).  Every shift ends at the FP64 true-residual
 * bound.  iters: all operator applications (multi-shift iterations plus
 * refinement iterations); refine_iters: the refinement part. */
int susy_b200_dev_congrad_multi_learned(susy_b200_lattice *h, susy_b200_net *net,
                                        const void *src, void *const *psim, int norder,
                                        const double *shift, int MaxCG, double errormin,
                                        int nrefine, double loose, double *size_r, int *iters,
                                        int *refine_iters);

/* Independent lattices at once (no reference counterpart: the reference
 * runs one lattice per process): one update() per handle, h[i] with r[i]
 * into res[i], the handles' streams driven concurrently by `threads` host
 * threads (at most n).  Every handle must launch on a stream of its own:
 * two handles on one stream (the same handle twice, or streams set to one
 * stream by susy_b200_set_stream) return SUSY_B200_EINVAL before any work,
 * since one thread's graph capture on a stream would take in the other
 * thread's launches.  Each handle's operator kernels are tuned first, one
 * handle at a time, unless already tuned.  Each lattice's result is the one
 * update() gives it alone.
 * Returns the total CG iterations or the first negative error code. */
int susy_b200_update_batch(susy_b200_lattice *const *h, const susy_b200_rhmc *const *r,
                           susy_b200_traj *res, int n, int threads);

/* dst[i] = (D^dag D + fmass_i^2) src[i] on lattice h[i], for n independent
 * lattices in two persistent launches over one work table of (lattice,
 * 128-site tile, output component) items instead of two launches per
 * lattice (no reference counterpart: the reference applies DSq,
 * utilities.c:874, to one lattice per process).  1 <= n <= 64 handles of
 * one NCOL on one device; lattice sizes, couplings and the RESCALE setting
 * may differ.  src[i] and dst[i] are device fields of h[i] in precision
 * prec (64 or 32).  Launches on cuda_stream (NULL: h[0]'s stream), after
 * the work already queued on every handle's stream, which in turn waits
 * for the launches, so the call is ordered like each handle's own
 * susy_b200_dev_DSq.  Each lattice's result is the one the site-major
 * table-driven kernels give it alone.  Uses (and on first use allocates)
 * each handle's DSq scratch field. */
#define SUSY_B200_BATCH_MAX 64
int susy_b200_DSq_batch(susy_b200_lattice *const *h, const void *const *src, void *const *dst,
                        int n, int prec, void *cuda_stream);
/* congrad_multi (susy/congrad_multi.c:26) for n independent lattices at
 * once, FP64, the reference's recurrences in their per-iteration form (the
 * solve susy_b200_cg_blocked(h, 0) selects for one lattice): lattice i
 * solves (D^dag D + fmass_i^2 + shift[i][j]) psim[i][j] = src[i] for
 * j < norder[i], each iteration being six launches for all lattices (the
 * batched operator of susy_b200_DSq_batch, D^dag with the dot product in its
 * epilogue, the recurrences one block per lattice, the vector updates over
 * one table of blocks).  Each lattice stops at its own iteration, as it
 * would alone; size_r[i] and iters[i] (either may be NULL) receive its final
 * |r|^2 and iterations.  No counterpart in the reference, which solves one
 * lattice per process.  1 <= n <= 64 distinct handles of one NCOL on one
 * device; src[i] and psim[i][j] are FP64 device fields of h[i].  Launches on
 * cuda_stream (NULL: h[0]'s stream) after the work queued on every handle's
 * stream, and returns once the solves are done.  Uses each handle's solver
 * state and scratch fields.  Returns the largest iteration count or a
 * negative error code. */
int susy_b200_dev_congrad_multi_batch(susy_b200_lattice *const *h, const void *const *src,
                                      void *const *const *psim, const int *norder,
                                      const double *const *shift, int n, int MaxCG,
                                      double errormin, double *size_r, int *iters,
                                      void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* SUSY_B200_H */
