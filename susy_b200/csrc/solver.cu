// Host drivers of the device-resident solvers (cg.cu kernels).
//
// multishift_fp64   the reference's congrad_multi in FP64 throughout.
// multishift_mixed  (1) the same multi-shift recurrences with the FP32
//                   operator and FP32 search/residual vectors, solutions
//                   accumulated in FP64, down to the FP32 noise floor;
//                   (2) per shift, FP64 true residual r = b - (D^dag D +
//                   sigma) x; while |r|^2 > errormin |b|^2, an FP32 CG on
//                   (D^dag D + sigma) e = r (zero guess) and x += e in FP64
//                   (defect correction with FP64 reliable updates).
//                   Every shift ends at the same FP64 true residual bound
//                   as the FP64 path requires.
#include <algorithm>
#include <cmath>
#include <vector>
#include "lattice.h"
#include "hmc.h"

namespace susy {

void* sol_field(susy_b200_lattice* h, int j) {
  while ((int)h->sols.size() <= j) h->sols.push_back(dalloc(h, field_bytes(h, NTF, 64)));
  return h->sols[j];
}

static void* pvec(susy_b200_lattice* h, int j, int prec) {
  std::vector<void*>& v = prec == 64 ? h->pvec64 : h->pvec32;
  while ((int)v.size() <= j) v.push_back(dalloc(h, field_bytes(h, NTF, prec)));
  return v[j];
}

static int* poll_words(susy_b200_lattice* h) {
  if (!h->poll) {
    if (cudaMallocHost(&h->poll, 4 * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      h->poll = nullptr;
    }
  }
  return h->poll;
}

// Multi-shift CG: operator and p/r/mp in precision pv, solutions in px.
// src is in precision pv.
static int ms_run(susy_b200_lattice* h, const void* src, void* const* psim, int norder,
                  const double* shift, int MaxCG, double errormin, int pv, int px,
                  double* size_r, int* iters) {
  cudaStream_t s = h->stream;
  const long n = tf_complex(h);
  const size_t bv = field_bytes(h, NTF, pv), bx = field_bytes(h, NTF, px);
  void* p0 = scratch_tf(h, 3, pv);
  void* r = scratch_tf(h, 4, pv);
  void* mp = scratch_tf(h, 5, pv);
  void* tmp = scratch_tf(h, 0, pv);
  double* part0 = partials(h, 0);
  double* part1 = partials(h, 1);
  int* pw = poll_words(h);
  if (!p0 || !r || !mp || !tmp || !part0 || !part1 || !pw) return set_err(h, SUSY_B200_ENOMEM);

  MsVecs v;
  v.p[0] = p0;
  v.psi[0] = psim[0];
  for (int j = 1; j < norder; j++) {
    v.p[j] = pvec(h, j, pv);
    if (!v.p[j]) return set_err(h, SUSY_B200_ENOMEM);
    v.psi[j] = psim[j];
  }
  v.r = r;
  v.mp = mp;

  // r = src, p0 = p_j = src, psi_j = 0   (congrad_multi.c:47-57)
  cudaMemcpyAsync(r, src, bv, cudaMemcpyDeviceToDevice, s);
  for (int j = 0; j < norder; j++) {
    cudaMemcpyAsync(v.p[j], src, bv, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(psim[j], 0, bx, s);
  }
  int ns = norder;
  cudaMemcpyAsync(&h->ms->nshift, &ns, sizeof(int), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(h->ms->shift, shift, sizeof(double) * norder, cudaMemcpyHostToDevice, s);
  ms_init(h->ms, src, pv, n, part0, MaxCG, errormin, s);

  const double fm2 = h->prm.fmass > 1e-8 ? h->prm.fmass * h->prm.fmass : 0.0;
  const int np_vec = vec_blocks(n);
  const int* skip = &h->ms->skip;
  const int chunk = 16;
  int launched = 0;
  for (;;) {
    for (int k = 0; k < chunk; k++) {
      dev_fop(h, p0, tmp, 1, pv, nullptr, 0.0, nullptr, skip);
      const int np_fop = dev_fop(h, tmp, mp, -1, pv, p0, fm2 + shift[0], part0, skip);
      ms_scalars1(h->ms, part0, np_fop, s);
      ms_update_fused(h->ms, v, pv, px, n, part1, s);
      ms_scalars2(h->ms, part1, np_vec, s);
      ms_update_p0(h->ms, v, pv, n, s);
    }
    launched += chunk;
    cudaMemcpyAsync(pw, &h->ms->skip, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!ck(h, cudaStreamSynchronize(s))) return SUSY_B200_ECUDA;
    if (pw[0] || launched >= MaxCG + chunk) break;
  }
  double rsq = 0.0;
  int it = 0;
  cudaMemcpyAsync(&rsq, &h->ms->rsq, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&it, &h->ms->iter, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (!ck(h, cudaStreamSynchronize(s))) return SUSY_B200_ECUDA;
  if (!(rsq == rsq)) return set_err(h, SUSY_B200_ENAN);
  if (size_r) *size_r = rsq;
  if (iters) *iters = it;
  return SUSY_B200_OK;
}

static void* ring_field(susy_b200_lattice* h, int q) {
  while ((int)h->ring.size() <= q) h->ring.push_back(dalloc(h, field_bytes(h, NTF, 64)));
  return h->ring[q];
}

// FP64 multi-shift CG with the blocked solution / search-vector update
// (cg.cu k_msb_block): the reference's recurrences and stopping rules,
// the shifted vectors touched once per MS_BLK iterations.
static int ms_run_block(susy_b200_lattice* h, const void* src, void* const* psim, int norder,
                        const double* shift, int MaxCG, double errormin, double* size_r,
                        int* iters) {
  cudaStream_t s = h->stream;
  const long n = tf_complex(h);
  const size_t bv = field_bytes(h, NTF, 64);
  void* p0 = scratch_tf(h, 3, 64);
  void* mp = scratch_tf(h, 5, 64);
  void* tmp = scratch_tf(h, 0, 64);
  double* part0 = partials(h, 0);
  double* part1 = partials(h, 1);
  int* pw = poll_words(h);
  if (!p0 || !mp || !tmp || !part0 || !part1 || !pw) return set_err(h, SUSY_B200_ENOMEM);
  MsBlockVecs v;
  for (int q = 0; q <= MS_BLK; q++) {
    v.ring[q] = ring_field(h, q);
    if (!v.ring[q]) return set_err(h, SUSY_B200_ENOMEM);
  }
  for (int j = 0; j < norder; j++) {
    v.P[j] = pvec(h, j, 64);
    if (!v.P[j]) return set_err(h, SUSY_B200_ENOMEM);
    v.x[j] = psim[j];
  }
  v.p0 = p0;
  v.mp = mp;
  // r(0) = src, p0 = P_j = src, psi_j = 0   (congrad_multi.c:47-57)
  cudaMemcpyAsync(v.ring[0], src, bv, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(p0, src, bv, cudaMemcpyDeviceToDevice, s);
  for (int j = 0; j < norder; j++) {
    cudaMemcpyAsync(v.P[j], src, bv, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(psim[j], 0, bv, s);
  }
  int ns = norder;
  cudaMemcpyAsync(&h->ms->nshift, &ns, sizeof(int), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(h->ms->shift, shift, sizeof(double) * norder, cudaMemcpyHostToDevice, s);
  ms_init(h->ms, src, 64, n, part0, MaxCG, errormin, s, 1);

  const double fm2 = h->prm.fmass > 1e-8 ? h->prm.fmass * h->prm.fmass : 0.0;
  const int np_vec = vec_blocks(n);
  const int* skip = &h->ms->skip;
  const int chunk = 2 * MS_BLK;
  int launched = 0;
  for (;;) {
    for (int k = 0; k < chunk; k++) {
      dev_fop(h, p0, tmp, 1, 64, nullptr, 0.0, nullptr, skip);
      const int np_fop = dev_fop(h, tmp, mp, -1, 64, p0, fm2 + shift[0], part0, skip);
      ms_scalars1(h->ms, part0, np_fop, s);
      msb_update_r(h->ms, v, n, part1, s);
      ms_scalars2(h->ms, part1, np_vec, s);
      msb_update_p0(h->ms, v, n, s);
      if ((k + 1) % MS_BLK == 0) msb_block(h->ms, v, n, s);
    }
    launched += chunk;
    cudaMemcpyAsync(pw, &h->ms->skip, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!ck(h, cudaStreamSynchronize(s))) return SUSY_B200_ECUDA;
    if (pw[0] || launched >= MaxCG + chunk) break;
  }
  double rsq = 0.0;
  int it = 0;
  cudaMemcpyAsync(&rsq, &h->ms->rsq, sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&it, &h->ms->iter, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (!ck(h, cudaStreamSynchronize(s))) return SUSY_B200_ECUDA;
  if (!(rsq == rsq)) return set_err(h, SUSY_B200_ENAN);
  if (size_r) *size_r = rsq;
  if (iters) *iters = it;
  return SUSY_B200_OK;
}

// Reference-faithful FP64 multi-shift CG (congrad_multi.c:26-221)
int multishift_fp64(susy_b200_lattice* h, const void* src, void* const* psim, int norder,
                    const double* shift, int MaxCG, double errormin, double* size_r,
                    int* iters) {
  if (h->ms_blocked)
    return ms_run_block(h, src, psim, norder, shift, MaxCG, errormin, size_r, iters);
  return ms_run(h, src, psim, norder, shift, MaxCG, errormin, 64, 64, size_r, iters);
}

static void* refine_field(susy_b200_lattice* h, int i, int prec) {
  while ((int)h->refine.size() <= 2 * i + 1) h->refine.push_back(nullptr);
  void** slot = &h->refine[2 * i + (prec == 64 ? 0 : 1)];
  if (!*slot) *slot = dalloc(h, field_bytes(h, NTF, prec));
  return *slot;
}

// |b - (D^dag D + fmass^2 + sigma) x|^2 with r64/r32 receiving the residual
static double true_residual(susy_b200_lattice* h, const void* b, const void* x, double sigma,
                            void* r64, void* r32) {
  const double fm2 = h->prm.fmass > 1e-8 ? h->prm.fmass * h->prm.fmass : 0.0;
  void* t = scratch_tf(h, 0, 64);
  void* ax = refine_field(h, 2, 64);
  double* part = partials(h, 2);
  dev_fop(h, x, t, 1, 64, nullptr, 0.0, nullptr, nullptr);
  dev_fop(h, t, ax, -1, 64, x, fm2 + sigma, nullptr, nullptr);
  const int nb = residual_partials(tf_complex(h), b, ax, r64, r32, part, h->stream);
  return host_sum(h, part, nb, 0);
}

int multishift_mixed(susy_b200_lattice* h, const void* src, void* const* psim, int norder,
                     const double* shift, int MaxCG, double errormin, double* size_r,
                     int* iters) {
  const long n = tf_complex(h);
  void* src32 = refine_field(h, 0, 32);
  void* r32 = refine_field(h, 1, 32);
  void* e32 = refine_field(h, 3, 32);
  if (!src32 || !r32 || !e32) return set_err(h, SUSY_B200_ENOMEM);
  convert_field(n, src, 64, src32, 32, h->stream);
  // (1) FP32 multi-shift pass; FP32 resolves |r|/|b| to ~1e-6
  const double floor32 = 1e-12;
  int it1 = 0, total = 0, rc;
  double sr = 0.0;
  rc = ms_run(h, src32, psim, norder, shift, MaxCG, std::max(errormin, floor32), 32, 64, &sr,
              &it1);
  if (rc) return rc;
  total += it1;
  // (2) FP64 true residuals and defect correction per shift
  double* part = partials(h, 2);
  if (!part) return set_err(h, SUSY_B200_ENOMEM);
  const double bnorm = [&] {
    norm2_partials(src, 64, n, part, h->stream);
    return host_sum(h, part, vec_blocks(n), 0);
  }();
  const double target = errormin * bnorm;
  double worst = 0.0;
  for (int j = 0; j < norder; j++) {
    double rr = true_residual(h, src, psim[j], shift[j], nullptr, r32);
    for (int outer = 0; outer < 12 && rr > target; outer++) {
      // inner FP32 CG to the remaining factor, capped at the FP32 floor
      const double want = std::max(0.25 * target / rr, floor32);
      void* e[1] = {e32};
      int it2 = 0;
      double s2 = 0.0;
      rc = ms_run(h, r32, e, 1, &shift[j], std::max(MaxCG - total, 1), want, 32, 32, &s2, &it2);
      if (rc) return rc;
      total += it2;
      add_low(n, e32, psim[j], h->stream);
      rr = true_residual(h, src, psim[j], shift[j], nullptr, r32);
      if (total >= MaxCG) break;
    }
    worst = std::max(worst, rr);
  }
  if (!ck(h, cudaGetLastError())) return SUSY_B200_ECUDA;
  if (!(worst == worst)) return set_err(h, SUSY_B200_ENAN);
  if (size_r) *size_r = worst;
  if (iters) *iters = total;
  return SUSY_B200_OK;
}

}  // namespace susy
