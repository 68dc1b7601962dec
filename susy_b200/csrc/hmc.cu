// C ABI of the forces, link update, actions, random fields and the HMC
// trajectory (reference susy/update_o.c, update_h.c, det_force.c,
// action.c, grsource.c).  Fields stay on the device for the whole
// trajectory; the host only sums FP64 block partials in a fixed order and
// takes the Metropolis decision.
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>
#include "lattice.h"
#include "hmc.h"

namespace susy {

static const double LAMBDA = 0.193, TWO_LAMBDA = 0.386, LAMBDA_MID = 0.614;  // defines.h:16-18

static long mat5(const susy_b200_lattice* h) { return 5L * h->N * h->N * h->g.S; }

// Sum n device partials on the host in index order (deterministic)
double host_sum(susy_b200_lattice* h, const double* dpart, int n, int offset) {
  std::vector<double> buf(n);
  if (!ck(h, cudaMemcpyAsync(buf.data(), dpart + offset, n * sizeof(double),
                             cudaMemcpyDeviceToHost, h->stream)))
    return NAN;
  if (!ck(h, cudaStreamSynchronize(h->stream))) return NAN;
  double s = 0.0;
  for (int i = 0; i < n; i++) s += buf[i];
  return s;
}

double* big_partials(susy_b200_lattice* h) {
  if (!h->bigpart) {
    const long n = 16L * h->N * h->N * h->g.S;
    const long nb = std::max<long>(force_blocks(h->g) * 2, (n + 255) / 256) + 8 * site_blocks(h->g);
    h->bigpart = (double*)dalloc(h, nb * sizeof(double));
    h->bigpart_n = nb;
  }
  return h->bigpart;
}

// U(N) generators Lambda_j (setup_lambda.c:10-64) on the device
static const void* generators(susy_b200_lattice* h) {
  if (h->gen) return h->gen;
  const int N = h->N, dimf = N * N;
  std::vector<double> L((size_t)dimf * N * N * 2, 0.0);
  auto at = [&](int j, int a, int b) -> double* { return &L[(((size_t)j * N + a) * N + b) * 2]; };
  const double s2 = 1.0 / std::sqrt(2.0);
  int count = 0;
  for (int i = 0; i < N; i++)
    for (int j = i + 1; j < N; j++) {
      at(count, i, j)[1] += s2;      // i / sqrt 2
      at(count + 1, i, j)[0] += s2;  // 1 / sqrt 2
      at(count, j, i)[1] += s2;
      at(count + 1, j, i)[0] -= s2;
      count += 2;
    }
  for (int i = 0; i < N - 1; i++) {
    const int j = N * (N - 1) + i, k = i + 1;
    const double v = 1.0 / std::sqrt(k * (k + 1.0));
    for (int l = 0; l <= k; l++) {
      at(j, l, l)[0] = 0.0;
      at(j, l, l)[1] = v;
    }
    at(j, k, k)[1] = -k * v;
  }
  for (int a = 0; a < N; a++)
    for (int b = 0; b < N; b++) at(dimf - 1, a, b)[0] = at(dimf - 1, a, b)[1] = 0.0;
  for (int i = 0; i < N; i++) at(dimf - 1, i, i)[1] = std::sqrt(1.0 / N);
  h->gen = dalloc(h, L.size() * sizeof(double));
  if (!h->gen) return nullptr;
  cudaMemcpyAsync(h->gen, L.data(), L.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  return h->gen;
}

static void* prn_state(susy_b200_lattice* h) {
  if (!h->prn) {
    h->prn = dalloc(h, 10L * h->g.S * sizeof(uint32_t));
    h->rng_bad = (int*)dalloc(h, sizeof(int));
    if (h->prn) init_prn(h->g, h->prm.iseed, h->prn, h->stream);
  }
  return h->prn;
}

// ---- host node generator (ranstuff.c:22-63), index = volume --------------
void node_prn_init(HostPrn& p, int seed, int index) {
  uint32_t sd = (uint32_t)seed;
  const uint32_t m = 69607u + 8u * (uint32_t)index;
  for (int k = 0; k < 7; k++) {
    sd = m * sd + 12345u;
    p.r[k] = (sd >> 8) & 0xffffffu;
  }
  sd = m * sd + 12345u;
  p.mult = 100005u + 8u * (uint32_t)index;
  p.add = 12345u;
  p.ic = sd;
}

double node_myrand(HostPrn& p) {
  const uint32_t t = (((p.r[5] >> 7) | (p.r[6] << 17)) ^ ((p.r[4] >> 1) | (p.r[5] << 23))) & 0xffffffu;
  for (int k = 6; k > 0; k--) p.r[k] = p.r[k - 1];
  p.r[0] = t;
  p.ic = p.ic * p.mult + p.add;
  return (double)(t ^ ((p.ic >> 8) & 0xffffffu)) * (1.0 / 16777216.0);
}

// ---- device-level pieces ---------------------------------------------------
int dev_update_u(susy_b200_lattice* h, double eps) {
  axpy_field(mat5(h), eps, h->mom, h->U, h->stream);
  return refresh_derived(h);
}

int dev_gauge_force(susy_b200_lattice* h, double eps, int det_only, double* norm) {
  double* part = big_partials(h);
  if (!part) return SUSY_B200_ENOMEM;
  const int nb = gauge_force(h->g, h->N, h->U, h->Uinv, h->pd, h->zw, h->D, h->F, h->mom, h->G,
                             h->prm.bmass, h->prm.kappa, h->prm.kappa_u1, eps, det_only, part,
                             h->stream);
  if (!ck(h, cudaGetLastError())) return SUSY_B200_ECUDA;
  if (norm) {
    const double n1 = host_sum(h, part, nb, 0);
    const double n2 = host_sum(h, part, nb, nb);
    if (det_only)
      *norm = n2;
    else
      *norm = eps * std::sqrt(h->prm.kappa * h->prm.kappa * n1 + n2) / h->g.V;
  }
  return h->err ? h->err : SUSY_B200_OK;
}

int dev_fermion_force(susy_b200_lattice* h, double eps, void* const* sol, int norder,
                      const double* amp4, double* norm) {
  void* psol = scratch_tf(h, 2, 64);
  double* part = big_partials(h);
  if (!psol || !part) return SUSY_B200_ENOMEM;
  cudaMemsetAsync(h->force, 0, field_bytes(h, 5, 64), h->stream);
  for (int n = 0; n < norder; n++) {
    dev_fop(h, sol[n], psol, 1, 64, nullptr, 0.0, nullptr, nullptr);
    fermion_force_pole(h->g, h->N, h->U, h->Uinv, h->pd, sol[n], psol, h->force, amp4[n], h->G,
                       h->stream);
  }
  const int nb = mom_sub(mat5(h), h->force, h->mom, eps, part, h->stream);
  if (!ck(h, cudaGetLastError())) return SUSY_B200_ECUDA;
  if (norm) *norm = eps * std::sqrt(host_sum(h, part, nb, 0)) / h->g.V;
  return h->err ? h->err : SUSY_B200_OK;
}

// parts: gauge, bmass, det, mom
int dev_action_bosonic(susy_b200_lattice* h, double* parts) {
  double* part = big_partials(h);
  if (!part) return SUSY_B200_ENOMEM;
  const int nb = action_partials(h->g, h->N, h->U, h->D, h->F, h->pd, h->mom, part, h->stream);
  if (!ck(h, cudaGetLastError())) return SUSY_B200_ECUDA;
  std::vector<double> buf(4L * nb);
  cudaMemcpyAsync(buf.data(), part, buf.size() * sizeof(double), cudaMemcpyDeviceToHost,
                  h->stream);
  if (!ck(h, cudaStreamSynchronize(h->stream))) return SUSY_B200_ECUDA;
  double s[4] = {0, 0, 0, 0};
  for (int k = 0; k < 4; k++)
    for (int i = 0; i < nb; i++) s[k] += buf[(size_t)k * nb + i];
  parts[0] = h->prm.kappa * s[0];
  parts[1] = h->prm.bmass > 1e-8 ? h->prm.kappa * h->prm.bmass * h->prm.bmass * s[1] : 0.0;
  parts[2] = h->prm.kappa_u1 > 1e-8 ? h->prm.kappa_u1 * s[2] : 0.0;
  parts[3] = s[3];
  return SUSY_B200_OK;
}

int dev_fermion_action(susy_b200_lattice* h, const void* src, void* const* sol, int norder,
                       const double* amp4, double ampdeg4, double* out) {
  double* part = big_partials(h);
  if (!part) return SUSY_B200_ENOMEM;
  if (!h->ptrbuf) {
    h->ptrbuf = dalloc(h, 2 * MS_MAXS * sizeof(void*));
    if (!h->ptrbuf) return SUSY_B200_ENOMEM;
  }
  std::vector<char> blob(2 * MS_MAXS * sizeof(void*), 0);
  memcpy(blob.data(), sol, norder * sizeof(void*));
  memcpy(blob.data() + MS_MAXS * sizeof(void*), amp4, norder * sizeof(double));
  cudaMemcpyAsync(h->ptrbuf, blob.data(), blob.size(), cudaMemcpyHostToDevice, h->stream);
  const long n = 16L * h->N * h->N * h->g.S;
  const int nb = fermion_action_partials(
      n, src, norder, (const void* const*)h->ptrbuf,
      (const double*)((char*)h->ptrbuf + MS_MAXS * sizeof(void*)), ampdeg4, part, h->stream);
  if (!ck(h, cudaGetLastError())) return SUSY_B200_ECUDA;
  *out = host_sum(h, part, nb, 0);
  return h->err ? h->err : SUSY_B200_OK;
}

int dev_ranmom(susy_b200_lattice* h) {
  const void* gen = generators(h);
  void* st = prn_state(h);
  if (!gen || !st) return SUSY_B200_ENOMEM;
  gauss_fill(h->g, h->N, st, gen, 5, 0, h->mom, h->rng_bad, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int dev_gaussian_tf(susy_b200_lattice* h, void* out) {
  const void* gen = generators(h);
  void* st = prn_state(h);
  if (!gen || !st) return SUSY_B200_ENOMEM;
  gauss_fill(h->g, h->N, st, gen, 16, 1, out, h->rng_bad, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

static void* field(susy_b200_lattice* h, std::vector<void*>& v, int i, int K) {
  while ((int)v.size() <= i) v.push_back(dalloc(h, field_bytes(h, K, 64)));
  return v[i];
}

// smdmom (grsource.c:13-40): mom <- c1 mom + c2 G, G drawn as ranmom draws
// it from the per-site generators
int dev_smdmom(susy_b200_lattice* h, double eps, double friction) {
  const double c1 = friction < 0.0 ? 0.0 : std::exp(-eps * friction);
  const double c2 = std::sqrt(1.0 - c1 * c1);
  void* keep = field(h, h->extra5, 2, 5);
  if (!keep) return SUSY_B200_ENOMEM;
  const size_t b5 = field_bytes(h, 5, 64);
  cudaMemcpyAsync(keep, h->mom, b5, cudaMemcpyDeviceToDevice, h->stream);
  int rc = dev_ranmom(h);
  if (rc) return rc;
  scale_field(mat5(h), c2, h->mom, h->stream);
  axpy_field(mat5(h), c1, keep, h->mom, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

// Solve with the configured solver; returns iterations (>= 0) or error
int solve(susy_b200_lattice* h, const susy_b200_rhmc* r, const void* src, void* const* psim,
          const double* shifts) {
  int it = 0;
  double sr = 0.0;
  int rc;
  if (r->solver == SUSY_B200_SOLVER_MIXED)
    rc = multishift_mixed(h, src, psim, r->Norder, shifts, r->niter, r->rsqmin, &sr, &it);
  else
    rc = multishift_fp64(h, src, psim, r->Norder, shifts, r->niter, r->rsqmin, &sr, &it);
  return rc ? rc : it;
}

// The Nroot pseudofermion solves of one force evaluation
// (update_o.c:169-176, 98-100, 111-113).  With two or more pseudofermions
// the odd ones run on the handle's second solver context (solver_shadow:
// own stream, scratch and solver state; links and derived fields shared)
// from a second host thread while this thread runs the even ones, so two
// multi-shift solves overlap on the GPU and each one's single-block scalar
// kernels and launch gaps fill with the other's operator kernels.  Each
// solve is the same kernel sequence on the same data either way: the
// solutions are identical to solving one after the other.  Returns the
// summed iterations or an error.
static int solve_pfs(susy_b200_lattice* h, const susy_b200_rhmc* r,
                     const std::vector<void*>& gsrc, std::vector<std::vector<void*>>& psim,
                     const double* shifts) {
  const int Nroot = r->Nroot;
  susy_b200_lattice* c = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (Nroot > 1 && h->pf_streams) {
    // the operator autotuner times kernels: it runs before the solves overlap
    if (h->fop_variant[0] < 0) autotune_fop(h, 64);
    if (r->solver == SUSY_B200_SOLVER_MIXED && h->fop_variant[1] < 0) autotune_fop(h, 32);
    c = solver_shadow(h);
    if (c && (cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) != cudaSuccess ||
              cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess)) {
      cudaGetLastError();
      c = nullptr;
    }
  }
  int total = 0;
  if (c) {
    // the context's stream starts after everything issued on the handle's
    cudaEventRecord(ev[0], h->stream);
    cudaStreamWaitEvent(c->stream, ev[0], 0);
    int odd_total = 0, odd_rc = 0, even_rc = 0;
    bool threaded = true;
    auto odd = [&]() {
      for (int n = 1; n < Nroot; n += 2) {
        const int it = solve(c, r, gsrc[n], psim[n].data(), shifts);
        if (it < 0) {
          odd_rc = it;
          return;
        }
        odd_total += it;
      }
    };
    std::thread t;
    try {
      t = std::thread(odd);
    } catch (...) {
      threaded = false;
    }
    for (int n = 0; n < Nroot && !even_rc; n += 2) {
      const int it = solve(h, r, gsrc[n], psim[n].data(), shifts);
      if (it < 0)
        even_rc = it;
      else
        total += it;
    }
    if (threaded)
      t.join();
    else
      odd();
    // and the handle's stream continues after the context's solves
    cudaEventRecord(ev[1], c->stream);
    cudaStreamWaitEvent(h->stream, ev[1], 0);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (even_rc) return even_rc;
    if (odd_rc) return set_err(h, odd_rc);
    return total + odd_total;
  }
  for (int n = 0; n < Nroot; n++) {
    const int it = solve(h, r, gsrc[n], psim[n].data(), shifts);
    if (it < 0) return it;
    total += it;
  }
  return total;
}

int dev_grsource(susy_b200_lattice* h, const susy_b200_rhmc* r, void* src, int* iters) {
  int rc = dev_gaussian_tf(h, src);
  if (rc) return rc;
  std::vector<void*> ps(r->Norder);
  for (int j = 0; j < r->Norder; j++)
    if (!(ps[j] = field(h, h->gr_psim, j, 16))) return SUSY_B200_ENOMEM;
  const int it = solve(h, r, src, ps.data(), r->shift8);
  if (it < 0) return it;
  if (iters) *iters = it;
  // src = ampdeg8 R + sum_j amp8[j] psim[j]   (grsource.c:293-297)
  const long n = 16L * h->N * h->N * h->g.S;
  scale_field(n, r->ampdeg8, src, h->stream);
  for (int j = 0; j < r->Norder; j++) axpy_field(n, r->amp8[j], ps[j], src, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

// smdgrsource (grsource.c:74-197): the fresh source of grsource, mixed
// with the previous one as src <- c2 fresh + c1 src.  The reference holds
// c1 and c2 in ints (grsource.c:79), so c1 = (int) exp(-traj_length
// friction) is 1 for friction == 0 and 0 otherwise (0 also for friction <
// 0), and c2 = (int) sqrt(1 - c1^2): the source is kept for friction == 0
// and fresh for every other friction.  The gaussian draws and the shift8 CG
// run either way, as in the reference.
static int dev_smdgrsource(susy_b200_lattice* h, const susy_b200_rhmc* r, void* src, void* old,
                           int* iters) {
  const int c1 = r->friction < 0.0 ? 0 : (int)std::exp(-r->traj_length * r->friction);
  const int c2 = (int)std::sqrt(1.0 - (double)(c1 * c1));
  cudaMemcpyAsync(old, src, field_bytes(h, NTF, 64), cudaMemcpyDeviceToDevice, h->stream);
  int rc = dev_grsource(h, r, src, iters);
  if (rc) return rc;
  const long n = 16L * h->N * h->N * h->g.S;
  if (c2 != 1) scale_field(n, (double)c2, src, h->stream);
  if (c1 != 0) axpy_field(n, (double)c1, old, src, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

static int action_total(susy_b200_lattice* h, const susy_b200_rhmc* r, void* const* gsrc,
                        void* const* const* psim, double* parts, double* total) {
  double b[4];
  int rc = dev_action_bosonic(h, b);
  if (rc) return rc;
  double t = b[0] + b[1] + b[2];
  double fsum = 0.0;
  for (int n = 0; n < r->Nroot; n++) {
    double f = 0.0;
    if ((rc = dev_fermion_action(h, gsrc[n], psim[n], r->Norder, r->amp4, r->ampdeg4, &f)))
      return rc;
    fsum += f;
  }
  t += fsum + b[3];
  if (parts) {
    parts[0] = b[0];
    parts[1] = b[1];
    parts[2] = b[2];
    parts[3] = fsum;
    parts[4] = b[3];
  }
  *total = t;
  return SUSY_B200_OK;
}

static int gauge_step(susy_b200_lattice* h, const susy_b200_rhmc* r, double eps, double* out) {
  // update_gauge_step, update_o.c:42-61
  const int n = r->nsteps[1];
  double norm = 0.0, x = 0.0;
  int rc = dev_gauge_force(h, eps * LAMBDA, 0, &x);
  if (rc) return rc;
  norm += x;
  for (int i = 1; i <= n; i++) {
    if ((rc = dev_update_u(h, 0.5 * eps))) return rc;
    if ((rc = dev_gauge_force(h, eps * LAMBDA_MID, 0, &x))) return rc;
    norm += x;
    if ((rc = dev_update_u(h, 0.5 * eps))) return rc;
    if ((rc = dev_gauge_force(h, eps * (i < n ? TWO_LAMBDA : LAMBDA), 0, &x))) return rc;
    norm += x;
  }
  *out = norm / n;
  return SUSY_B200_OK;
}

int dev_update(susy_b200_lattice* h, const susy_b200_rhmc* r, susy_b200_traj* res,
               const double* mom_in, const double* const* src_in) {
  if (r->Nroot < 1 || r->Nroot > SUSY_B200_MAX_NROOT || r->Norder < 1 || r->Norder > MS_MAXS ||
      (r->algorithm != SUSY_B200_HMC && r->algorithm != SUSY_B200_SMD))
    return set_err(h, SUSY_B200_EINVAL);
  const int Nroot = r->Nroot, Norder = r->Norder;
  std::vector<void*> gsrc(Nroot);
  std::vector<std::vector<void*>> psim(Nroot, std::vector<void*>(Norder));
  std::vector<void* const*> pp(Nroot);
  for (int n = 0; n < Nroot; n++) {
    if (!(gsrc[n] = field(h, h->gsrc, n, 16))) return SUSY_B200_ENOMEM;
    for (int j = 0; j < Norder; j++)
      if (!(psim[n][j] = field(h, h->traj_psim, n * MS_MAXS + j, 16))) return SUSY_B200_ENOMEM;
    pp[n] = psim[n].data();
  }
  void* old_U = field(h, h->extra5, 0, 5);
  void* old_mom = field(h, h->extra5, 1, 5);
  if (!old_U || !old_mom) return SUSY_B200_ENOMEM;
  memset(res, 0, sizeof(*res));
  int iters = 0, rc, it;

  // ranmom / smdmom (update_o.c:149-154) and pseudofermion sources
  // (update_o.c:159-165)
  const bool smd = r->algorithm == SUSY_B200_SMD;
  if ((rc = smd ? dev_smdmom(h, r->traj_length, r->friction) : dev_ranmom(h))) return rc;
  if (mom_in && (rc = upload_links(h, h->mom, mom_in, 0, 5))) return rc;
  for (int n = 0; n < Nroot; n++) {
    if (smd) {
      void* old = field(h, h->gsrc, SUSY_B200_MAX_NROOT + n, 16);
      if (!old) return SUSY_B200_ENOMEM;
      rc = dev_smdgrsource(h, r, gsrc[n], old, &it);
    } else {
      rc = dev_grsource(h, r, gsrc[n], &it);
    }
    if (rc) return rc;
    iters += it;
  }
  if (src_in)
    for (int n = 0; n < Nroot; n++)
      if ((rc = susy_b200_tf_upload(h, gsrc[n], 64, src_in[n]))) return rc;
  // psim = (D^dag D + shift4)^-1 gsrc   (update_o.c:169-176)
  if ((it = solve_pfs(h, r, gsrc, psim, r->shift4)) < 0) return it;
  iters += it;
  double start = 0.0, end = 0.0;
  if ((rc = action_total(h, r, gsrc.data(), pp.data(), res->start_parts, &start))) return rc;
  const size_t b5 = field_bytes(h, 5, 64);
  cudaMemcpyAsync(old_U, h->U, b5, cudaMemcpyDeviceToDevice, h->stream);
  cudaMemcpyAsync(old_mom, h->mom, b5, cudaMemcpyDeviceToDevice, h->stream);

  // update_step (update_o.c:67-121)
  const double f_eps = r->traj_length / (double)r->nsteps[0];
  const double g_eps = f_eps / (2.0 * r->nsteps[1]);
  double gnorm = 0.0, max_gf = 0.0, x;
  std::vector<double> fnorm(Nroot, 0.0), max_ff(Nroot, 0.0);
  auto ff = [&](int n, double eps) -> int {
    double t = 0.0;
    int e = dev_fermion_force(h, eps, psim[n].data(), Norder, r->amp4, &t);
    fnorm[n] += t;
    if (t > max_ff[n]) max_ff[n] = t;
    return e;
  };
  for (int n = 0; n < Nroot; n++)
    if ((rc = ff(n, f_eps * LAMBDA))) return rc;
  for (int i = 1; i <= r->nsteps[0]; i++) {
    if ((rc = gauge_step(h, r, g_eps, &x))) return rc;
    gnorm += x;
    if (x > max_gf) max_gf = x;
    if ((it = solve_pfs(h, r, gsrc, psim, r->shift4)) < 0) return it;
    iters += it;
    for (int n = 0; n < Nroot; n++)
      if ((rc = ff(n, f_eps * LAMBDA_MID))) return rc;
    if ((rc = gauge_step(h, r, g_eps, &x))) return rc;
    gnorm += x;
    if (x > max_gf) max_gf = x;
    if ((it = solve_pfs(h, r, gsrc, psim, r->shift4)) < 0) return it;
    iters += it;
    for (int n = 0; n < Nroot; n++)
      if ((rc = ff(n, f_eps * (i < r->nsteps[0] ? TWO_LAMBDA : LAMBDA)))) return rc;
  }
  if ((rc = action_total(h, r, gsrc.data(), pp.data(), res->end_parts, &end))) return rc;
  double change = end - start;
  if (!(std::fabs(change) <= 1e20)) change = 1.0e20;  // update_o.c:219-226
  const double xr = node_myrand(h->node_prn);
  const int accept = r->no_metropolis ? 1 : !(std::exp(-change) < xr);
  if (!accept && r->traj_length > 0.0) {
    cudaMemcpyAsync(h->U, old_U, b5, cudaMemcpyDeviceToDevice, h->stream);
    // reverse momenta (update_o.c:236-238)
    cudaMemsetAsync(h->mom, 0, b5, h->stream);
    axpy_field(mat5(h), -1.0, old_mom, h->mom, h->stream);
    if ((rc = refresh_derived(h))) return rc;
  }
  int bad = 0;
  cudaMemcpyAsync(&bad, h->rng_bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (!ck(h, cudaStreamSynchronize(h->stream))) return SUSY_B200_ECUDA;
  res->delta_S = change;
  res->start_S = start;
  res->end_S = end;
  res->accept = accept;
  res->iters = iters;
  res->xrandom = xr;
  res->gnorm = gnorm / (2.0 * r->nsteps[0]);
  res->max_gf = max_gf;
  for (int n = 0; n < Nroot; n++) {
    res->fnorm[n] = fnorm[n] / (2.0 * r->nsteps[0]);
    res->max_ff[n] = max_ff[n];
  }
  if (bad) return set_err(h, SUSY_B200_ENAN);
  if (!(start == start) || !(end == end)) return set_err(h, SUSY_B200_ENAN);
  return iters;
}

}  // namespace susy

using namespace susy;

extern "C" {

int susy_b200_update_u(susy_b200_lattice* h, double eps) {
  if (!h) return SUSY_B200_EINVAL;
  return dev_update_u(h, eps);
}

int susy_b200_gauge_force(susy_b200_lattice* h, double eps, double* norm) {
  if (!h) return SUSY_B200_EINVAL;
  return dev_gauge_force(h, eps, 0, norm);
}

int susy_b200_det_force(susy_b200_lattice* h, double eps, double* norm) {
  if (!h) return SUSY_B200_EINVAL;
  return dev_gauge_force(h, eps, 1, norm);
}

int susy_b200_fermion_force(susy_b200_lattice* h, double eps, const double* src,
                            const double* const* sol, int norder, const double* amp4,
                            double* norm) {
  (void)src;  // the reference's fermion_force ignores src as well (update_h.c:928-978)
  if (!h || !sol || !amp4 || norder < 1 || norder > MS_MAXS) return set_err(h, SUSY_B200_EINVAL);
  std::vector<void*> ps(norder);
  for (int j = 0; j < norder; j++) {
    ps[j] = sol_field(h, j);
    if (!ps[j]) return SUSY_B200_ENOMEM;
    int rc = susy_b200_tf_upload(h, ps[j], 64, sol[j]);
    if (rc) return rc;
  }
  return dev_fermion_force(h, eps, ps.data(), norder, amp4, norm);
}

int susy_b200_dev_fermion_force(susy_b200_lattice* h, double eps, void* const* sol, int norder,
                                const double* amp4, double* norm) {
  if (!h || !sol || !amp4 || norder < 1 || norder > MS_MAXS) return set_err(h, SUSY_B200_EINVAL);
  return dev_fermion_force(h, eps, sol, norder, amp4, norm);
}

int susy_b200_action(susy_b200_lattice* h, int nroot, const double* const* src,
                     const double* const* sol, int norder, const double* amp4, double ampdeg4,
                     double* parts) {
  if (!h || !parts || nroot < 0 || (nroot > 0 && (!src || !sol || !amp4)) || norder > MS_MAXS)
    return set_err(h, SUSY_B200_EINVAL);
  double b[4];
  int rc = dev_action_bosonic(h, b);
  if (rc) return rc;
  parts[0] = b[0];
  parts[1] = b[1];
  parts[2] = b[2];
  parts[4] = b[3];
  double fsum = 0.0;
  void* s = scratch_tf(h, 1, 64);
  std::vector<void*> ps(norder);
  for (int j = 0; j < norder; j++)
    if (!(ps[j] = sol_field(h, j))) return SUSY_B200_ENOMEM;
  for (int n = 0; n < nroot; n++) {
    if ((rc = susy_b200_tf_upload(h, s, 64, src[n]))) return rc;
    for (int j = 0; j < norder; j++)
      if ((rc = susy_b200_tf_upload(h, ps[j], 64, sol[(size_t)n * norder + j]))) return rc;
    double f = 0.0;
    if ((rc = dev_fermion_action(h, s, ps.data(), norder, amp4, ampdeg4, &f))) return rc;
    fsum += f;
  }
  parts[3] = fsum;
  return SUSY_B200_OK;
}

int susy_b200_seed(susy_b200_lattice* h, int iseed) {
  if (!h) return SUSY_B200_EINVAL;
  h->prm.iseed = iseed;
  void* st = prn_state(h);
  if (!st) return SUSY_B200_ENOMEM;
  init_prn(h->g, iseed, st, h->stream);
  node_prn_init(h->node_prn, iseed, h->g.V);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_ranmom(susy_b200_lattice* h) {
  if (!h) return SUSY_B200_EINVAL;
  return dev_ranmom(h);
}

int susy_b200_smdmom(susy_b200_lattice* h, double eps, double friction) {
  if (!h) return SUSY_B200_EINVAL;
  return dev_smdmom(h, eps, friction);
}

int susy_b200_grsource(susy_b200_lattice* h, const susy_b200_rhmc* r, double* src) {
  if (!h || !r || !src) return set_err(h, SUSY_B200_EINVAL);
  void* d = scratch_tf(h, 1, 64);
  if (!d) return SUSY_B200_ENOMEM;
  int it = 0;
  int rc = dev_grsource(h, r, d, &it);
  if (rc) return rc;
  rc = susy_b200_tf_download(h, d, 64, src);
  return rc ? rc : it;
}

int susy_b200_gaussian_tf(susy_b200_lattice* h, double* out) {
  if (!h || !out) return set_err(h, SUSY_B200_EINVAL);
  void* d = scratch_tf(h, 1, 64);
  if (!d) return SUSY_B200_ENOMEM;
  int rc = dev_gaussian_tf(h, d);
  return rc ? rc : susy_b200_tf_download(h, d, 64, out);
}

int susy_b200_update(susy_b200_lattice* h, const susy_b200_rhmc* r, susy_b200_traj* res) {
  if (!h || !r || !res) return set_err(h, SUSY_B200_EINVAL);
  return dev_update(h, r, res, nullptr, nullptr);
}

int susy_b200_update_replay(susy_b200_lattice* h, const susy_b200_rhmc* r, susy_b200_traj* res,
                            const double* mom, const double* const* src) {
  if (!h || !r || !res) return set_err(h, SUSY_B200_EINVAL);
  return dev_update(h, r, res, mom, src);
}

}  // extern "C"
