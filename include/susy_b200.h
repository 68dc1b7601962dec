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
int susy_b200_sync(susy_b200_lattice *h);
int susy_b200_volume(const susy_b200_lattice *h);

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
int susy_b200_dev_DSq(susy_b200_lattice *h, const void *src, void *dst, int prec);
int susy_b200_dev_congrad_multi(susy_b200_lattice *h, const void *src, void *const *psim,
                                int norder, const double *shift, int MaxCG, double errormin,
                                double *size_r, int *iters);

#ifdef __cplusplus
}
#endif
#endif /* SUSY_B200_H */
