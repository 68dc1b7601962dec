/*
 * b200_shim.c -- the reference-side binding of libsusy_b200 for a 4d_Q16
 * SUSY LATTICE build (per-call drop-in at the function boundary).
 *
 * A reference build adds this file to 4d_Q16/susy/ and takes these
 * functions from it instead of from its own objects:
 *   fermion_op, DSq        susy/utilities.c:765, :874
 *   congrad_multi          susy/congrad_multi.c:26
 *   fermion_force          susy/update_h.c:928
 *   gauge_force            susy/update_h.c:15 (det_force included when
 *                          kappa_u1 > 0, as update_h.c:257 calls it)
 *   update_u               susy/update_o.c:20
 * Everything else -- setup, the RHMC driver update() and its Metropolis
 * step, grsource, ranmom, the actions and every measurement of control.c --
 * stays the reference's own code and calls these through their usual
 * names.  The reference keeps its globals (lattice[], Norder, shift[],
 * amp4[], couplings); the shim hands them to one library handle.  Links and
 * momenta are read from and written back to lattice[] in place, with the
 * site stride sizeof(site), so the host view stays exact after every call.
 *
 * oracle/build_ref.sh (target shim) links it into the reference's own
 * susy_hmc: the replaced symbols are made weak in the reference's objects
 * (objcopy --weaken-symbol on objects compiled here from the unmodified
 * sources), so these strong definitions take their place at link time.
 */
#include "susy_includes.h"
#include "susy_b200.h"

static susy_b200_lattice *H = NULL;

static void b200_check(int rc) {
  if (rc < 0) {
    node0_printf("susy_b200: %s\n", susy_b200_error_string(rc));
    terminate(1);
  }
}

static void b200_init(void) {
  susy_b200_params p;
  if (H)
    return;
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  p.nt = nt;
  p.ncol = NCOL;
  p.pbc = (int)PBC;
  p.kappa = kappa;
  p.bmass = bmass;
  p.fmass = fmass;
  p.kappa_u1 = kappa_u1;
  p.G = G;
  p.iseed = iseed;
  p.device = 0;
  H = susy_b200_create(&p);
  if (H == NULL) {
    node0_printf("susy_b200_create failed\n");
    terminate(1);
  }
#ifdef RESCALE
  /* the build's RESCALE (defines.h:30) doubles eta in and out of fermion_op */
  b200_check(susy_b200_set_rescale(H, 1));
#endif
  node0_printf("susy_b200: hot path on the GPU (libsusy_b200)\n");
}

#define LINKS ((double *)&lattice[0].link[0])
#define MOM ((double *)&lattice[0].mom[0])

static void b200_links(void) {
  b200_init();
  b200_check(susy_b200_set_links(H, LINKS, sizeof(site)));
}

void fermion_op(Twist_Fermion *src, Twist_Fermion *dest, int sign) {
  b200_links();
  if (susy_b200_fermion_op(H, (const double *)src, (double *)dest, sign) == SUSY_B200_EINVAL) {
    node0_printf("Error: incorrect sign in fermion_op: %d\n", sign);
    terminate(1);
  }
}

void DSq(Twist_Fermion *src, Twist_Fermion *dest) {
  b200_links();
  b200_check(susy_b200_DSq(H, (const double *)src, (double *)dest));
}

int congrad_multi(Twist_Fermion *src, Twist_Fermion **psim, int MaxCG, Real errormin,
                  Real *size_r) {
  double sr = 0.0;
  int it;
  b200_links();
  it = susy_b200_congrad_multi(H, (const double *)src, (double *const *)psim, Norder, shift,
                               MaxCG, errormin, &sr);
  b200_check(it);
  total_iters += it;            /* congrad_multi.c:80 counts every iteration */
  *size_r = sr;
  return it;
}

double fermion_force(Real eps, Twist_Fermion *src, Twist_Fermion **sol) {
  double norm = 0.0;
  b200_links();
  b200_check(susy_b200_set_mom(H, MOM, sizeof(site)));
  b200_check(susy_b200_fermion_force(H, eps, (const double *)src, (const double *const *)sol,
                                     Norder, amp4, &norm));
  b200_check(susy_b200_get_mom(H, MOM, sizeof(site)));
  return norm;
}

double gauge_force(Real eps) {
  double norm = 0.0;
  b200_links();
  b200_check(susy_b200_set_mom(H, MOM, sizeof(site)));
  b200_check(susy_b200_gauge_force(H, eps, &norm));
  b200_check(susy_b200_get_mom(H, MOM, sizeof(site)));
  return norm;
}

void update_u(Real eps) {
  b200_links();
  b200_check(susy_b200_set_mom(H, MOM, sizeof(site)));
  b200_check(susy_b200_update_u(H, eps));
  b200_check(susy_b200_get_links(H, LINKS, sizeof(site)));
  /* the reference's own derived fields feed its actions and measurements:
     refresh them as update_o.c:31-34 does after every link update */
  compute_plaqdet();
  compute_Uinv();
  compute_DmuUmu();
  compute_Fmunu();
}
