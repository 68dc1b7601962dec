// Host driver of the device-resident multi-shift CG (cg.cu kernels).
#include <algorithm>
#include <vector>
#include "lattice.h"

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

// Reference-faithful FP64 multi-shift CG (congrad_multi.c:26-221)
int multishift_fp64(susy_b200_lattice* h, const void* src, void* const* psim, int norder,
                    const double* shift, int MaxCG, double errormin, double* size_r,
                    int* iters) {
  cudaStream_t s = h->stream;
  const long n = tf_complex(h);
  const size_t bytes = field_bytes(h, NTF, 64);
  void* p0 = scratch_tf(h, 3, 64);
  void* r = scratch_tf(h, 4, 64);
  void* mp = scratch_tf(h, 5, 64);
  void* tmp = scratch_tf(h, 0, 64);
  double* part0 = partials(h, 0);
  double* part1 = partials(h, 1);
  int* pw = poll_words(h);
  if (!p0 || !r || !mp || !tmp || !part0 || !part1 || !pw) return set_err(h, SUSY_B200_ENOMEM);

  MsVecs v;
  v.p[0] = p0;
  v.psi[0] = psim[0];
  for (int j = 1; j < norder; j++) {
    v.p[j] = pvec(h, j, 64);
    if (!v.p[j]) return set_err(h, SUSY_B200_ENOMEM);
    v.psi[j] = psim[j];
  }
  v.r = r;
  v.mp = mp;

  // r = src, p0 = p_j = src, psi_j = 0
  cudaMemcpyAsync(r, src, bytes, cudaMemcpyDeviceToDevice, s);
  for (int j = 0; j < norder; j++) {
    cudaMemcpyAsync(v.p[j], src, bytes, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(psim[j], 0, bytes, s);
  }
  // shifts into the device state
  MsState hs;
  std::fill((char*)&hs, (char*)&hs + sizeof(hs), 0);
  hs.nshift = norder;
  for (int j = 0; j < norder; j++) hs.shift[j] = shift[j];
  // nshift and shift[] are the only host-provided members; init fills the rest
  cudaMemcpyAsync(&h->ms->nshift, &hs.nshift, sizeof(int), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(h->ms->shift, hs.shift, sizeof(double) * norder, cudaMemcpyHostToDevice, s);
  ms_init(h->ms, src, 64, n, part0, MaxCG, errormin, s);

  const double fm2 = h->prm.fmass > 1e-8 ? h->prm.fmass * h->prm.fmass : 0.0;
  const int np_fop = fop_partials(h->g);
  const int np_vec = vec_blocks(n);
  const int* skip = &h->ms->skip;
  const int chunk = 16;
  int launched = 0;
  for (;;) {
    for (int k = 0; k < chunk; k++) {
      dev_fop(h, p0, tmp, 1, 64, nullptr, 0.0, nullptr, skip);
      dev_fop(h, tmp, mp, -1, 64, p0, fm2 + shift[0], part0, skip);
      ms_scalars1(h->ms, part0, np_fop, s);
      ms_update_a(h->ms, v, 64, n, part1, s);
      ms_scalars2(h->ms, part1, np_vec, s);
      ms_update_b(h->ms, v, 64, n, s);
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

}  // namespace susy
