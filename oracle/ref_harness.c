/*
 * C harness around the UNMODIFIED reference CPU code (4d_Q16/susy).
 *
 * TEST INFRASTRUCTURE ONLY.  build_ref.sh compiles this file together with
 * the reference's own objects (everything of susy_hmc except control.o) into
 * oracle/_ref/libsusyref_n<NCOL>.so.  Tests, the golden-vector generator and
 * bench.py's CPU leg load that library with ctypes to (a) pin the numpy
 * restatement in oracle/susy_np.py and (b) time the reference's own
 * DSq / congrad_multi / fermion_force on the host.  Nothing shipped in
 * susy_b200/ links or loads it.
 *
 * Set-up mirrors 4d_Q16/susy/control.c:16-29 (setup, setup_lambda, epsilon,
 * setup_PtoP, setup_FQ, setup_rhmc, readin) by feeding the reference its
 * own key/value input through stdin.  Field exchange is flat doubles in the
 * reference's memory order: sites in node_index order
 * (generic/layout_hyper_prime.c:157), each site's Twist_Fermion
 * {Fsite, Flink[5], Fplaq[10]} (susy/lattice.h:18-22) of e[NCOL][NCOL]
 * {re, im}.
 *
 * The reference keeps all state in globals and appends gather tables on
 * every set-up, so one process holds one lattice: callers spawn a fresh
 * process per configuration.
 */
#define CONTROL
#include "susy_includes.h"
#include <unistd.h>
#include <fcntl.h>

/* Reference functions that susy_includes.h does not declare */
double bmass_action(void);
double det_action(void);
double fermion_action(Twist_Fermion *src, Twist_Fermion **sol);
double mom_action(void);
double update_gauge_step(Real eps);

#define MAT_DOUBLES (2 * NCOL * NCOL)
#define TF_DOUBLES (16 * MAT_DOUBLES)

static int h_ready = 0;
static int saved_stdout = -1;

int ref_ncol(void) { return NCOL; }
int ref_tf_doubles(void) { return TF_DOUBLES; }

/* Redirect the reference's stdout chatter to a file ("" restores it) */
void ref_redirect_stdout(const char *path) {
  fflush(stdout);
  if (path && path[0]) {
    int fd = open(path, O_WRONLY | O_CREAT | O_APPEND, 0644);
    if (fd < 0)
      return;
    if (saved_stdout < 0)
      saved_stdout = dup(1);
    dup2(fd, 1);
    close(fd);
  }
  else if (saved_stdout >= 0) {
    dup2(saved_stdout, 1);
    close(saved_stdout);
    saved_stdout = -1;
  }
}

/* Run the reference set-up on a key/value input file (control.c:16-47) */
int ref_init(const char *input_path) {
  int argc = 1, prompt;
  char *argv0 = "ref_harness", **argv = &argv0;
  if (h_ready)
    return -1;
  if (freopen(input_path, "r", stdin) == NULL)
    return -2;
  initialize_machine(&argc, &argv);
  g_sync();
  prompt = setup();
  setup_lambda();
  epsilon();
  setup_PtoP();
  setup_FQ();
  setup_rhmc();
  if (readin(prompt) != 0)
    return -3;
  h_ready = 1;
  return sites_on_node;
}

int ref_volume(void) { return volume; }

/* Coordinates x, y, z, t of every site in node_index order */
void ref_site_coords(int *xyzt) {
  int i;
  site *s;
  FORALLSITES(i, s) {
    xyzt[4 * i + 0] = s->x;
    xyzt[4 * i + 1] = s->y;
    xyzt[4 * i + 2] = s->z;
    xyzt[4 * i + 3] = s->t;
  }
}

/* Per-site RNG state (ranstuff.c:22): r0..r6, multiplier, addend, ic_state */
void ref_site_prn(unsigned long *out) {
  int i;
  site *s;
  FORALLSITES(i, s) {
    unsigned long *o = out + 10 * i;
    o[0] = s->site_prn.r0; o[1] = s->site_prn.r1; o[2] = s->site_prn.r2;
    o[3] = s->site_prn.r3; o[4] = s->site_prn.r4; o[5] = s->site_prn.r5;
    o[6] = s->site_prn.r6; o[7] = s->site_prn.multiplier;
    o[8] = s->site_prn.addend; o[9] = s->site_prn.ic_state;
  }
}

void ref_node_prn(unsigned long *o) {
  o[0] = node_prn.r0; o[1] = node_prn.r1; o[2] = node_prn.r2;
  o[3] = node_prn.r3; o[4] = node_prn.r4; o[5] = node_prn.r5;
  o[6] = node_prn.r6; o[7] = node_prn.multiplier;
  o[8] = node_prn.addend; o[9] = node_prn.ic_state;
}

static void copy_site_mats(double *out, size_t member_offset, int nmat,
                           int to_host) {
  int i;
  site *s;
  size_t bytes = (size_t)nmat * sizeof(matrix);
  FORALLSITES(i, s) {
    char *p = (char *)s + member_offset;
    if (to_host)
      memcpy(out + (size_t)i * nmat * MAT_DOUBLES, p, bytes);
    else
      memcpy(p, out + (size_t)i * nmat * MAT_DOUBLES, bytes);
  }
}

void ref_get_links(double *out) { copy_site_mats(out, F_OFFSET(link[0]), NUMLINK, 1); }
void ref_set_links(double *in) { copy_site_mats(in, F_OFFSET(link[0]), NUMLINK, 0); }
void ref_get_mom(double *out) { copy_site_mats(out, F_OFFSET(mom[0]), NUMLINK, 1); }
void ref_set_mom(double *in) { copy_site_mats(in, F_OFFSET(mom[0]), NUMLINK, 0); }
void ref_get_fU(double *out) { copy_site_mats(out, F_OFFSET(f_U[0]), NUMLINK, 1); }

/* update_u's derived fields (update_o.c:31-34) */
void ref_compute_all(void) {
  compute_plaqdet();
  compute_Uinv();
  compute_DmuUmu();
  compute_Fmunu();
}

/* plaqdet[a][b] for all a != b, as [V][5][5] complex (diagonal zero) */
void ref_get_plaqdet(double *out) {
  int i, a, b;
  site *s;
  FORALLSITES(i, s) {
    for (a = 0; a < NUMLINK; a++)
      for (b = 0; b < NUMLINK; b++) {
        double *o = out + 2 * ((size_t)i * 25 + a * 5 + b);
        o[0] = (a == b) ? 0.0 : plaqdet[a][b][i].real;
        o[1] = (a == b) ? 0.0 : plaqdet[a][b][i].imag;
      }
  }
}

void ref_get_DmuUmu(double *out) {
  int i;
  site *s;
  FORALLSITES(i, s)
    memcpy(out + (size_t)i * MAT_DOUBLES, &DmuUmu[i], sizeof(matrix));
}

void ref_get_Fmunu(double *out) {
  int i, p;
  site *s;
  FORALLSITES(i, s)
    for (p = 0; p < NPLAQ; p++)
      memcpy(out + ((size_t)i * NPLAQ + p) * MAT_DOUBLES, &Fmunu[p][i],
             sizeof(matrix));
}

void ref_get_Uinv(double *out) {
  int i, a;
  site *s;
  FORALLSITES(i, s)
    for (a = 0; a < NUMLINK; a++)
      memcpy(out + ((size_t)i * NUMLINK + a) * MAT_DOUBLES, &Uinv[a][i],
             sizeof(matrix));
}

/* Rational-approximation tables chosen by setup_rhmc (setup_rhmc.c:2000) */
int ref_rhmc(double *amp4_, double *shift4_, double *amp8_, double *shift8_,
             double *degs) {
  int j;
  for (j = 0; j < Norder; j++) {
    amp4_[j] = amp4[j];
    shift4_[j] = shift4[j];
    amp8_[j] = amp8[j];
    shift8_[j] = shift8[j];
  }
  degs[0] = ampdeg4;
  degs[1] = ampdeg8;
  return Norder;
}

void ref_fermion_op(double *src, double *dest, int sign) {
  fermion_op((Twist_Fermion *)src, (Twist_Fermion *)dest, sign);
}

void ref_DSq(double *src, double *dest) {
  DSq((Twist_Fermion *)src, (Twist_Fermion *)dest);
}

/* congrad_multi with caller-chosen shifts; psim is Norder contiguous fields */
/* congrad_multi on nshift shifts (1 <= nshift <= the setup's Norder): the
 * reference loops over the global Norder, so it is set to nshift for the
 * call and restored after it */
int ref_congrad_multi(double *src, double *psim, double *shifts, int nshift, int MaxCG,
                      double errormin, double *size_r, int *total) {
  int j, it, norder_setup = Norder;
  Real sr = 0.0;
  Twist_Fermion **ps;
  if (nshift < 1 || nshift > norder_setup)
    return -1;
  ps = malloc(sizeof(Twist_Fermion *) * nshift);
  for (j = 0; j < nshift; j++) {
    ps[j] = (Twist_Fermion *)(psim + (size_t)j * sites_on_node * TF_DOUBLES);
    shift[j] = shifts[j];
  }
  Norder = nshift;
  it = congrad_multi((Twist_Fermion *)src, ps, MaxCG, errormin, &sr);
  Norder = norder_setup;
  *size_r = sr;
  if (total)
    *total = total_iters;
  free(ps);
  return it;
}

double ref_fermion_force(double eps, double *src, double *sol) {
  int j;
  double r;
  Twist_Fermion **ps = malloc(sizeof(Twist_Fermion *) * Norder);
  for (j = 0; j < Norder; j++)
    ps[j] = (Twist_Fermion *)(sol + (size_t)j * sites_on_node * TF_DOUBLES);
  r = fermion_force(eps, (Twist_Fermion *)src, ps);
  free(ps);
  return r;
}

double ref_gauge_force(double eps) { return gauge_force(eps); }
double ref_det_force(double eps) { return det_force(eps); }
void ref_update_u(double eps) { update_u(eps); }
double ref_update_gauge_step(double eps) { return update_gauge_step(eps); }

/* Action pieces (action.c:106-286); out = {gauge, bmass, det, fermion, mom} */
void ref_action_parts(double *src, double *sol, double *out) {
  int j;
  Twist_Fermion **ps = malloc(sizeof(Twist_Fermion *) * Norder);
  for (j = 0; j < Norder; j++)
    ps[j] = (Twist_Fermion *)(sol + (size_t)j * sites_on_node * TF_DOUBLES);
  out[0] = gauge_action(NODET);
  out[1] = bmass > IMAG_TOL ? bmass_action() : 0.0;
  out[2] = kappa_u1 > IMAG_TOL ? det_action() : 0.0;
  out[3] = src ? fermion_action((Twist_Fermion *)src, ps) : 0.0;
  out[4] = mom_action();
  free(ps);
}

#ifndef SMD_ALGORITHM
void ref_ranmom(void) { ranmom(); }

int ref_grsource(double *src) { return grsource((Twist_Fermion *)src); }
#else
/* The SMD build's refreshes (grsource.c:13-40,74-197) */
void ref_smdmom(double eps) { smdmom(eps); }
#endif

int ref_update(void) { return update(); }

void ref_plaquette(double *ss, double *st) { plaquette(ss, st); }

/* Per-trajectory measurements of control.c:85-138 (the reference's own
 * functions; measure_det and widths print their results to stdout) */
void ref_ploop(int dir, int project, double *out) {
  double mod = 0.0;
  complex c = ploop(dir, project, &mod);
  out[0] = c.real; out[1] = c.imag; out[2] = mod;
}

double ref_link_trace(double *linktr, double *width, double *link_det, double *det_ave,
                      double *det_width) {
  return link_trace(linktr, width, link_det, det_ave, det_width);
}

void ref_scalar_eig(int project, double *ave, double *width, double *mn, double *mx) {
  scalar_eig(project, ave, width, mn, mx);
}

double ref_gauge_action(int do_det) { return gauge_action(do_det); }

void ref_measure_det(void) { measure_det(); fflush(stdout); }

void ref_widths(void) { widths(); fflush(stdout); }

/* Scalar globals a caller may need to mirror */
void ref_params(double *out) {
  out[0] = kappa; out[1] = bmass; out[2] = fmass; out[3] = kappa_u1;
  out[4] = G; out[5] = rsqmin; out[6] = traj_length; out[7] = nsteps[0];
  out[8] = nsteps[1]; out[9] = niter; out[10] = Nroot; out[11] = Norder;
  out[12] = PBC; out[13] = total_iters; out[14] = lambda;
}

void ref_set_total_iters(int n) { total_iters = n; }
