// Host drivers of the device-resident solvers (cg.cu kernels).
//
// multishift_fp64   the reference's congrad_multi in FP64 throughout.
// multishift_mixed  (1) the same multi-shift recurrences (blocked update)
//                   with the operator in FP32 once |r| < 3e-4 |src| and
//                   FP64 reliable updates of the base residual;
//                   (2) per shift, the FP64 true residual
//                   r = b - (D^dag D + sigma) x; a shift with
//                   |r|^2 > errormin |b|^2 gets CG passes on
//                   (D^dag D + sigma) e = r, x += e, with the FP32
//                   operator (FP64 once a pass gains under 10x).
//                   Every shift ends at or below the FP64 true residual
//                   bound errormin |b|^2.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "fop.cuh"
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
    if (cudaMallocHost(&h->poll, (4 + MS_MAXS) * sizeof(int)) != cudaSuccess) {
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

// Multi-shift CG (FP64, per-iteration form: ms_run) of nl independent
// lattices of one NCOL at once.  Every lattice is set up as ms_run sets up
// one solve (its own state, vectors and partials in its handle); then each
// iteration is six launches for all lattices together: the batched
// operator D, D^dag with the (fmass^2 + shift_0) p0 epilogue and the
// <p0, mp> partials, the first recurrences, the vector update with the
// |r|^2 partials, the second recurrences and the p0 update.  A lattice
// whose solve has stopped drops out of every launch through its stop flag;
// the host polls the flags every 16 iterations.  Launches go to st.
static int ms_run_batch(susy_b200_lattice* const* hs, int nl, const void* const* src,
                        void* const* const* psim, const int* norder,
                        const double* const* shift, int MaxCG, double errormin,
                        double* size_r, int* iters, cudaStream_t st) {
  std::vector<MsLat> L(nl);
  std::vector<FopArgs<double>> aD(nl), aDd(nl);
  int vtot = 0;
  for (int i = 0; i < nl; i++) {
    susy_b200_lattice* h = hs[i];
    const long n = tf_complex(h);
    const size_t bv = field_bytes(h, NTF, 64);
    void* p0 = scratch_tf(h, 3, 64);
    void* r = scratch_tf(h, 4, 64);
    void* mp = scratch_tf(h, 5, 64);
    void* tmp = scratch_tf(h, 0, 64);
    double* part0 = partials(h, 0);
    double* part1 = partials(h, 1);
    if (!p0 || !r || !mp || !tmp || !part0 || !part1) return SUSY_B200_ENOMEM;
    MsVecs v;
    v.p[0] = p0;
    v.psi[0] = psim[i][0];
    for (int j = 1; j < norder[i]; j++) {
      if (!(v.p[j] = pvec(h, j, 64))) return SUSY_B200_ENOMEM;
      v.psi[j] = psim[i][j];
    }
    v.r = r;
    v.mp = mp;
    // the allocations above zero their fields on h's stream
    if (h->stream != st && cudaStreamSynchronize(h->stream) != cudaSuccess) return SUSY_B200_ECUDA;
    // r = src, p0 = p_j = src, psi_j = 0   (congrad_multi.c:47-57)
    cudaMemcpyAsync(r, src[i], bv, cudaMemcpyDeviceToDevice, st);
    for (int j = 0; j < norder[i]; j++) {
      cudaMemcpyAsync(v.p[j], src[i], bv, cudaMemcpyDeviceToDevice, st);
      cudaMemsetAsync(psim[i][j], 0, bv, st);
    }
    const int ns = norder[i];
    cudaMemcpyAsync(&h->ms->nshift, &ns, sizeof(int), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(h->ms->shift, shift[i], sizeof(double) * ns, cudaMemcpyHostToDevice, st);
    ms_init(h->ms, src[i], 64, n, part0, MaxCG, errormin, st);
    const double fm2 = h->prm.fmass > 1e-8 ? h->prm.fmass * h->prm.fmass : 0.0;
    aD[i] = batch_fop_args<double>(h, p0, tmp, nullptr, 0.0, nullptr, &h->ms->skip);
    aDd[i] = batch_fop_args<double>(h, tmp, mp, p0, fm2 + shift[i][0], part0, &h->ms->skip);
    L[i].st = h->ms;
    L[i].v = v;
    L[i].n = n;
    L[i].part0 = part0;
    L[i].np0 = 16 * ((h->g.V + 127) / 128);
    L[i].part1 = part1;
    L[i].vblk0 = vtot;
    L[i].vblocks = vec_blocks(n);
    vtot += L[i].vblocks;
  }
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return SUSY_B200_ECUDA;
  }
  MsLat* dL = nullptr;
  int* dskip = nullptr;
  if (cudaMalloc(&dL, nl * sizeof(MsLat)) != cudaSuccess ||
      cudaMalloc(&dskip, nl * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dL);
    return SUSY_B200_ENOMEM;
  }
  cudaMemcpyAsync(dL, L.data(), nl * sizeof(MsLat), cudaMemcpyHostToDevice, st);
  const int N = hs[0]->N;
  std::vector<int> hskip(nl, 0);
  int rc = SUSY_B200_OK;
  const int chunk = 16;
  int launched = 0;
  for (;;) {
    for (int k = 0; k < chunk && !rc; k++) {
      if (fermion_op_batch<double>(aD.data(), nl, N, 1, sms, st) < 0 ||
          fermion_op_batch<double>(aDd.data(), nl, N, -1, sms, st) < 0)
        rc = SUSY_B200_EINVAL;
      ms_batch_scalars1(dL, nl, st);
      ms_batch_update_fused(dL, nl, vtot, st);
      ms_batch_scalars2(dL, nl, st);
      ms_batch_update_p0(dL, nl, vtot, st);
    }
    launched += chunk;
    ms_batch_skips(dL, nl, dskip, st);
    cudaMemcpyAsync(hskip.data(), dskip, nl * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = SUSY_B200_ECUDA;
    if (rc) break;
    bool all = true;
    for (int i = 0; i < nl; i++) all = all && hskip[i];
    if (all || launched >= MaxCG + chunk) break;
  }
  for (int i = 0; i < nl && !rc; i++) {
    double rsq = 0.0;
    int it = 0;
    cudaMemcpyAsync(&rsq, &hs[i]->ms->rsq, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&it, &hs[i]->ms->iter, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      rc = SUSY_B200_ECUDA;
      break;
    }
    if (!(rsq == rsq)) rc = SUSY_B200_ENAN;
    if (size_r) size_r[i] = rsq;
    if (iters) iters[i] = it;
  }
  cudaFree(dL);
  cudaFree(dskip);
  if (cudaGetLastError() != cudaSuccess && !rc) rc = SUSY_B200_ECUDA;
  return rc;
}

int multishift_batch(susy_b200_lattice* const* hs, int nl, const void* const* src,
                     void* const* const* psim, const int* norder, const double* const* shift,
                     int MaxCG, double errormin, double* size_r, int* iters, cudaStream_t st) {
  return ms_run_batch(hs, nl, src, psim, norder, shift, MaxCG, errormin, size_r, iters, st);
}

static void* ring_field(susy_b200_lattice* h, int q) {
  while ((int)h->ring.size() <= q) h->ring.push_back(dalloc(h, field_bytes(h, NTF, 64)));
  return h->ring[q];
}

// FP32 residual ring slots 0..MS_BLK of the mixed solver's FP32 phase
static void* vec32_field(susy_b200_lattice* h, int q) {
  while ((int)h->vec32.size() <= q) h->vec32.push_back(dalloc(h, field_bytes(h, NTF, 32)));
  return h->vec32[q];
}

// One captured chunk of solver iterations.  Capture is thread-local, so
// other host threads driving other lattices (susy_b200_update_batch) may
// keep launching meanwhile.  If capture or instantiation fails the chunk
// runs as plain launches.
struct ChunkGraph {
  cudaGraphExec_t exec = nullptr;
  long long kernels = 0;
  bool ready = false;
  template <typename F>
  void capture(susy_b200_lattice* h, int prec, F&& issue) {
    // the operator's autotuner synchronises: run it before capturing
    const int pi = prec == 64 ? 0 : 1;
    if (h->fop_variant[pi] < 0) autotune_fop(h, prec);
    cudaStream_t s = h->stream;
    const long long c0 = thread_launch_count();
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      h->use_graphs = 0;
      return;
    }
    issue();
    cudaGraph_t g = nullptr;
    const cudaError_t e1 = cudaStreamEndCapture(s, &g);
    kernels = thread_launch_count() - c0;
    count_launches(-kernels);   // captured, not launched
    if (e1 != cudaSuccess || !g || cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
      cudaGetLastError();
      if (g) cudaGraphDestroy(g);
      exec = nullptr;
      h->use_graphs = 0;
      return;
    }
    cudaGraphDestroy(g);
    ready = true;
  }
  void launch(cudaStream_t s) {
    cudaGraphLaunch(exec, s);
    count_launches(kernels);
  }
  ~ChunkGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

static void* refine_field(susy_b200_lattice* h, int i, int prec);
static double true_residual(susy_b200_lattice* h, const void* b, const void* x, double sigma,
                            void* r64, void* r32);

// Multi-shift CG with the blocked solution / search-vector update
// (cg.cu k_msb_block): the reference's recurrences and stopping rules,
// the shifted vectors touched once per MS_BLK iterations.
//
// mixed = false: FP64 throughout (the reference's solver).
// mixed = true: the operator runs in FP64 until |r| < mix_switch |src|
// (handle setting, default 3e-4) and in FP32 after that; with mix_vec32
// (off by default) the residual ring and the operator's input are FP32 fields
// from then on too, while the recurrences, the shifted search vectors and
// the solutions stay FP64.  Once the operator is FP32,
// the iterated residual drifts from the true one by the FP32 rounding of
// each product, so at block boundaries, whenever |r| fell by mix_reliable
// (default 1e-2) since the last check (or, with mix_interval > 0, every
// mix_interval iterations rounded up to a block) and when the solve stops,
// the FP64 true residual b - (D^dag D + sigma_0) psi_0 replaces it, with
// the same correction applied to the search vectors (a reliable update); the solve
// only ends when the true residual meets the stopping bound.  The FP32
// products enter only when the residual is small, so the shifted systems,
// which never see a residual replacement, keep an error of order FP32
// rounding times that residual.  Switching earlier costs more in the
// per-shift correction solves than it saves.  On the thermalised 12^3 x 24
// U(3) benchmark configuration (FP64: 3128 iterations) |r| stays near
// 1e-3 ... 1e-2 |src| for the first ~1700 iterations before it falls at
// ~130 iterations per decade, so the FP32 operator can only take the last
// ~40% of the solve: switching at 1e-3 took 4653 iterations in all, at
// 3e-4 3184 (1.11x faster than FP64), 1e-4 3175, 3e-5 3169, 1e-6 3157.

static int ms_run_block(susy_b200_lattice* h, const void* src, void* const* psim, int norder,
                        const double* shift, int MaxCG, double errormin, bool mixed,
                        double* size_r, int* iters, double errormin_base = -1.0,
                        const FrozenHook* on_frozen = nullptr) {
  cudaStream_t s = h->stream;
  const long n = tf_complex(h);
  const size_t bv = field_bytes(h, NTF, 64);
  void* p0 = scratch_tf(h, 3, 64);
  void* mp = scratch_tf(h, 5, 64);
  void* tmp = scratch_tf(h, 0, 64);
  void* p0_32 = mixed ? scratch_tf(h, 3, 32) : nullptr;
  void* mp32 = mixed ? scratch_tf(h, 5, 32) : nullptr;
  void* tmp32 = mixed ? scratch_tf(h, 0, 32) : nullptr;
  double* part0 = partials(h, 0);
  double* part1 = partials(h, 1);
  int* pw = poll_words(h);
  if (!p0 || !mp || !tmp || !part0 || !part1 || !pw || (mixed && (!p0_32 || !mp32 || !tmp32)))
    return set_err(h, SUSY_B200_ENOMEM);
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
  v.p0_32 = nullptr;
  v.mp32 = mp32;
  v.f32 = 0;
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
  if (errormin_base > 0.0) ms_set_stop(h->ms, errormin_base, s);

  const double fm2 = h->prm.fmass > 1e-8 ? h->prm.fmass * h->prm.fmass : 0.0;
  const int* skip = &h->ms->skip;
  // a fixed reliable-update schedule polls at every block boundary
  const int chunk = (mixed && h->mix_interval > 0) ? MS_BLK : 2 * MS_BLK;
  double* pd = (double*)(pw + 2);  // pinned: the iterated |r|^2
  bool fp32_op = false;
  double bnorm = 0.0, last_true = 0.0, rsqstop = 0.0;
  if (mixed) {
    cudaMemcpyAsync(pd, &h->ms->source_norm, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (!ck(h, cudaStreamSynchronize(s))) return SUSY_B200_ECUDA;
    bnorm = last_true = *pd;
    rsqstop = errormin * bnorm;
  }
  int launched = 0, replacements = 0, last_rel = 0;
  std::vector<char> handed(norder, 0);
  // SUSY_B200_CG_TRACE=1 prints the solver's progress at every poll (stderr)
  static const bool trace = [] {
    const char* e = getenv("SUSY_B200_CG_TRACE");
    return e && e[0] == '1';
  }();
  auto issue_chunk = [&]() {
    for (int k = 0; k < chunk; k++) {
      int np_fop;
      if (fp32_op) {
        dev_fop(h, p0_32, tmp32, 1, 32, nullptr, 0.0, nullptr, skip);
        np_fop = dev_fop(h, tmp32, mp32, -1, 32, p0_32, fm2 + shift[0], part0, skip);
      } else {
        dev_fop(h, p0, tmp, 1, 64, nullptr, 0.0, nullptr, skip);
        np_fop = dev_fop(h, tmp, mp, -1, 64, p0, fm2 + shift[0], part0, skip);
      }
      ms_scalars1(h->ms, part0, np_fop, s);
      msb_update_r(h->ms, v, n, part1, fp32_op, s);
      msb_update_p0(h->ms, v, n, s);
      if ((k + 1) % MS_BLK == 0) msb_block(h->ms, v, n, s);
    }
  };
  // Switch to the FP32 operator at iteration it (a block boundary, or the
  // start); false when a field cannot be allocated
  auto to_fp32 = [&](int it) -> bool {
    fp32_op = true;
    last_rel = it;
    convert_field(n, p0, 64, p0_32, 32, s);
    if (h->mix_vec32) {
      // FP32 residuals from here on (a block boundary, so the residual of
      // this iteration is the only ring slot the next steps read), and the
      // operator's input is the FP32 p0 itself.  The shifted search vectors
      // and the solutions stay FP64: rounding P_j to FP32 every block puts
      // an error of order u_32 |P_j| (not u_32 |r|) into every shifted
      // system, which measured 8x the per-shift correction iterations.
      const int slot = it % (MS_BLK + 1);
      for (int q = 0; q <= MS_BLK; q++)
        if (!vec32_field(h, q)) return false;
      convert_field(n, v.ring[slot], 64, vec32_field(h, slot), 32, s);
      for (int q = 0; q <= MS_BLK; q++) v.ring[q] = vec32_field(h, q);
      v.p0 = p0_32;
      v.f32 = 1;
    } else {
      // the operator input from now on: an FP32 copy of p0, kept by the p0
      // update
      v.p0_32 = p0_32;
    }
    return true;
  };
  // fp32_below = 1: the FP32 operator from the first iteration
  if (mixed && h->mix_switch >= 1.0 && !to_fp32(0)) return set_err(h, SUSY_B200_ENOMEM);
  // A chunk's ~100 launches are captured once per operator precision into a
  // CUDA graph and replayed: every argument of them is fixed for the solve
  // (the convergence test and the freezing of shifts read device state).
  ChunkGraph graphs[2];
  for (;;) {
    if (h->use_graphs) {
      ChunkGraph& cg = graphs[fp32_op ? 1 : 0];
      if (!cg.ready) cg.capture(h, fp32_op ? 32 : 64, issue_chunk);
      if (cg.ready)
        cg.launch(s);
      else
        issue_chunk();
    } else {
      issue_chunk();
    }
    launched += chunk;
    cudaMemcpyAsync(pw, &h->ms->skip, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(pw + 1, &h->ms->iter, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(pd, &h->ms->rsq, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (on_frozen)
      cudaMemcpyAsync(pw + 4, h->ms->converged, norder * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (!ck(h, cudaStreamSynchronize(s))) return SUSY_B200_ECUDA;
    // a shift frozen by now had its last block pass at this block boundary
    if (on_frozen)
      for (int j = 1; j < norder; j++)
        if (pw[4 + j] && !handed[j]) {
          handed[j] = 1;
          (*on_frozen)(j);
        }
    bool stop = pw[0] != 0;
    if (trace)
      fprintf(stderr, "susy_b200 cg: it %d rsq %.6e rel %.3e stop %d fp32 %d\n", pw[1], *pd,
              bnorm > 0 ? *pd / bnorm : 0.0, (int)stop, (int)fp32_op);
    if (mixed) {
      const double rsq = *pd;
      const int it = pw[1];
      const bool due = h->mix_interval > 0 ? it - last_rel >= h->mix_interval
                                            : rsq < h->mix_reliable * h->mix_reliable * last_true;
      if (!fp32_op && !stop && rsq < h->mix_switch * h->mix_switch * bnorm) {
        if (!to_fp32(it)) return set_err(h, SUSY_B200_ENOMEM);
      } else if (fp32_op && (stop || due)) {
        // reliable update at the block boundary: psi_0 is current
        void* rt64 = refine_field(h, 4, 64);
        if (!rt64) return set_err(h, SUSY_B200_ENOMEM);
        const double rt = true_residual(h, src, psim[0], shift[0], rt64, nullptr);
        if (trace) fprintf(stderr, "susy_b200 cg: reliable update at %d: true rsq %.6e\n", it, rt);
        if (!(rt == rt)) return set_err(h, SUSY_B200_ENAN);
        msb_replace(h->ms, v, n, rt64, rt, s);
        last_true = rt;
        last_rel = it;
        replacements++;
        stop = (rt <= rsqstop || it >= MaxCG);
      } else if (fp32_op && !(rsq <= 1e4 * last_true)) {
        // the FP32 recurrence left the true residual behind: give up (the
        // caller falls back to the FP64 solver)
        if (trace) fprintf(stderr, "susy_b200 cg: FP32 phase diverged at %d\n", it);
        return SUSY_B200_ENOCONV;
      }
    }
    if (stop || launched >= MaxCG + chunk) break;
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
                    int* iters, const FrozenHook* on_frozen) {
  if (h->ms_blocked)
    return ms_run_block(h, src, psim, norder, shift, MaxCG, errormin, false, size_r, iters,
                        -1.0, on_frozen);
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
                     int* iters, const FrozenHook* on_frozen, char* redo) {
  const long n = tf_complex(h);
  int it1 = 0, rc;
  double sr = 0.0;
  // (1) multi-shift pass, FP32 operator once the residual is small; should
  // the FP32 phase fail (a non-finite value, or the iterated residual
  // running away from the true one), the plain FP64 solve replaces it
  rc = ms_run_block(h, src, psim, norder, shift, MaxCG, errormin, true, &sr, &it1, -1.0,
                    on_frozen);
  if (rc == SUSY_B200_ENOCONV || rc == SUSY_B200_ENAN) {
    cudaStreamSynchronize(h->stream);
    h->err = 0;
    if (redo)
      for (int j = 0; j < norder; j++) redo[j] = 1;
    int it64 = 0;
    rc = ms_run_block(h, src, psim, norder, shift, MaxCG, errormin, false, &sr, &it64);
    it1 += it64;
  }
  if (rc) return rc;
  int total = it1;
  // (2) every shift's FP64 true residual; a shift above the bound (the FP32
  // products leave the shifted systems an error of order FP32 rounding
  // times the residual at the switch) gets correction solves
  // (D^dag D + sigma) e = r, x += e.  The correction only needs the leading
  // digits of e, so it runs with the FP32 operator and FP32 recurrences
  // (FP64 e), each pass asked for at most 1e-4 in |r| and the FP64 true
  // residual deciding after it (iterative refinement); a pass that gains
  // less than 10x in |r|^2 switches the shift's remaining passes to FP64.
  double* part = partials(h, 2);
  void* r64 = refine_field(h, 0, 64);
  void* r32 = refine_field(h, 0, 32);
  void* e64 = refine_field(h, 1, 64);
  if (!part || !r64 || !r32 || !e64) return set_err(h, SUSY_B200_ENOMEM);
  norm2_partials(src, 64, n, part, h->stream);
  const double bnorm = host_sum(h, part, vec_blocks(n), 0);
  const double target = errormin * bnorm;
  double worst = 0.0;
  for (int j = 0; j < norder; j++) {
    double rr = true_residual(h, src, psim[j], shift[j], r64, r32);
    bool fp32 = h->mix_correct32 != 0;
    for (int outer = 0; outer < 8 && rr > target && total < MaxCG; outer++) {
      void* e[1] = {e64};
      int it2 = 0;
      double s2 = 0.0;
      if (fp32)
        rc = ms_run(h, r32, e, 1, &shift[j], MaxCG - total, std::max(0.25 * target / rr, 1e-8),
                    32, 64, &s2, &it2);
      else
        rc = ms_run(h, r64, e, 1, &shift[j], MaxCG - total, 0.25 * target / rr, 64, 64, &s2,
                    &it2);
      if (rc) return rc;
      total += it2;
      if (redo) redo[j] = 1;
      axpy_field(n, 1.0, e64, psim[j], h->stream);
      const double before = rr;
      rr = true_residual(h, src, psim[j], shift[j], r64, r32);
      if (!(rr == rr)) return set_err(h, SUSY_B200_ENAN);
      if (fp32 && !(rr < 0.1 * before)) fp32 = false;
    }
    worst = std::max(worst, rr);
  }
  if (!ck(h, cudaGetLastError())) return SUSY_B200_ECUDA;
  if (!(worst == worst)) return set_err(h, SUSY_B200_ENAN);
  if (size_r) *size_r = worst;
  if (iters) *iters = total;
  return SUSY_B200_OK;
}

// Flexible CG (Notay's FCG with one previous direction) on
// (D^dag D + fmass^2 + sigma) x = b from the given x, preconditioned by the
// network (identity when net is null: then it is plain CG), in FP64, until
// |r|^2 <= target:
//   z = M(r); p = z - (<z, q_prev> / <p_prev, q_prev>) p_prev; q = A p;
//   alpha = <p, r> / <p, q>; x += alpha p; r -= alpha q.
// The recursive residual is checked against the true one at the end (and
// the iteration restarted from it once if the two disagree).
static int fcg_refine(susy_b200_lattice* h, susy_b200_net* net, const void* b, void* x,
                      double sigma, double target, int maxit, int* its) {
  cudaStream_t s = h->stream;
  const long n = tf_complex(h);
  const double fm2 = h->prm.fmass > 1e-8 ? h->prm.fmass * h->prm.fmass : 0.0;
  void* r = refine_field(h, 5, 64);
  void* z = refine_field(h, 6, 64);
  void* p = refine_field(h, 7, 64);
  void* q = refine_field(h, 8, 64);
  void* t = scratch_tf(h, 0, 64);
  double* part = partials(h, 2);
  if (!r || !z || !p || !q || !t || !part) return set_err(h, SUSY_B200_ENOMEM);
  const int nb = vec_blocks(n);
  auto dot = [&](const void* a, const void* c) {
    rdot_partials(n, a, c, part, s);
    return host_sum(h, part, nb, 0);
  };
  auto apply_A = [&](const void* in, void* out) {
    dev_fop(h, in, t, 1, 64, nullptr, 0.0, nullptr, nullptr);
    dev_fop(h, t, out, -1, 64, in, fm2 + sigma, nullptr, nullptr);
  };
  auto precond = [&](const void* in, void* out) -> int {
    if (net) return net_apply(net, in, out);
    copy_field(n, in, out, s);
    return SUSY_B200_OK;
  };
  int it = 0, rc;
  for (int restart = 0; restart < 2; restart++) {
    double rr = true_residual(h, b, x, sigma, r, nullptr);
    if (!(rr == rr)) return set_err(h, SUSY_B200_ENAN);
    if (rr <= target) break;
    if ((rc = precond(r, z))) return rc;
    copy_field(n, z, p, s);
    apply_A(p, q);
    while (it < maxit) {
      const double pq = dot(p, q);
      const double alpha = dot(p, r) / pq;
      axpy_field(n, alpha, p, x, s);
      axpy_field(n, -alpha, q, r, s);
      it++;
      norm2_partials(r, 64, n, part, s);
      rr = host_sum(h, part, nb, 0);
      if (!(rr == rr)) return set_err(h, SUSY_B200_ENAN);
      if (rr <= target) break;
      if ((rc = precond(r, z))) return rc;
      const double beta = -dot(z, q) / pq;
      scale_field(n, beta, p, s);
      axpy_field(n, 1.0, z, p, s);
      apply_A(p, q);
    }
    if (it >= maxit) break;
  }
  if (its) *its = it;
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

// Learned-preconditioned solve: the blocked FP64 multi-shift with the base
// (smallest) shift stopped at loose |src|^2 while the others keep freezing
// at errormin |src|^2; then every shift whose FP64 true residual is above
// errormin |src|^2 is refined by flexible CG, preconditioned by the network
// for the nrefine smallest shifts and unpreconditioned for the rest.
int multishift_learned(susy_b200_lattice* h, susy_b200_net* net, const void* src,
                       void* const* psim, int norder, const double* shift, int MaxCG,
                       double errormin, int nrefine, double loose, double* size_r, int* iters,
                       int* refine_iters) {
  int it1 = 0, rc;
  double sr = 0.0;
  rc = ms_run_block(h, src, psim, norder, shift, MaxCG, errormin, false, &sr, &it1, loose);
  if (rc) return rc;
  const long n = tf_complex(h);
  double* part = partials(h, 2);
  if (!part) return set_err(h, SUSY_B200_ENOMEM);
  norm2_partials(src, 64, n, part, h->stream);
  const double target = errormin * host_sum(h, part, vec_blocks(n), 0);
  int total = it1, refine = 0;
  double worst = 0.0;
  void* r64 = refine_field(h, 0, 64);
  if (!r64) return set_err(h, SUSY_B200_ENOMEM);
  for (int j = 0; j < norder; j++) {
    int its = 0;
    rc = fcg_refine(h, j < nrefine ? net : nullptr, src, psim[j], shift[j], target,
                    std::max(MaxCG - total, 1), &its);
    if (rc) return rc;
    total += its;
    refine += its;
    worst = std::max(worst, true_residual(h, src, psim[j], shift[j], r64, nullptr));
  }
  if (!(worst == worst)) return set_err(h, SUSY_B200_ENAN);
  if (size_r) *size_r = worst;
  if (iters) *iters = total;
  if (refine_iters) *refine_iters = refine;
  return SUSY_B200_OK;
}

}  // namespace susy
