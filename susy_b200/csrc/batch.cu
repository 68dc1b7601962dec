// Many independent lattices at once (susy_b200_update_batch): one RHMC
// trajectory per lattice, concurrently.  Each lattice handle owns its
// stream, fields and solver state, and its trajectory is the same host
// driver a single update() runs (hmc.cu), so the result of every lattice
// is bit for bit the one it gets alone.  A pool of host threads takes the
// lattices in turn; a small lattice's kernels occupy a few SMs, so with
// several lattices in flight their streams fill the GPU together.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>
#include "fop.cuh"
#include "lattice.h"

namespace susy {
int dev_update(susy_b200_lattice* h, const susy_b200_rhmc* r, susy_b200_traj* res,
               const double* mom_in, const double* const* src_in);
}

using namespace susy;

extern "C" int susy_b200_update_batch(susy_b200_lattice* const* hs,
                                      const susy_b200_rhmc* const* rs, susy_b200_traj* res,
                                      int n, int threads) {
  if (!hs || !rs || !res || n < 0) return SUSY_B200_EINVAL;
  for (int i = 0; i < n; i++)
    if (!hs[i] || !rs[i]) return SUSY_B200_EINVAL;
  // One stream per handle: a worker captures its solver chunks into CUDA
  // graphs, and a capture takes in every launch made to its stream, from
  // any thread, so a second lattice on the same stream would have its work
  // recorded into the first one's graph and its own syncs refused.
  {
    std::vector<cudaStream_t> st(n);
    for (int i = 0; i < n; i++) st[i] = hs[i]->stream;
    std::sort(st.begin(), st.end());
    if (std::adjacent_find(st.begin(), st.end()) != st.end()) return SUSY_B200_EINVAL;
  }
  // Every handle's operator kernels are tuned here, one handle after the
  // other on this thread with the GPU otherwise idle, before any worker
  // starts: tuned inside the workers, each handle would time its kernels
  // against the other lattices' work (noise for picks) and allocate its
  // tuning fields while other workers capture their solver graphs.
  for (int i = 0; i < n; i++) {
    if (cudaSetDevice(hs[i]->prm.device) != cudaSuccess) return SUSY_B200_ECUDA;
    for (int prec : {64, 32}) {
      if (hs[i]->fop_variant[prec == 64 ? 0 : 1] >= 0) continue;
      const int rt = autotune_fop(hs[i], prec);
      if (rt < 0) return rt;
    }
  }
  const int nt = std::max(1, std::min(threads > 0 ? threads : 1, n));
  std::atomic<int> next(0);
  std::vector<int> rc(n, 0);
  auto work = [&]() {
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= n) return;
      int dev = hs[i]->prm.device;
      cudaSetDevice(dev);
      rc[i] = dev_update(hs[i], rs[i], &res[i], nullptr, nullptr);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; t++) pool.emplace_back(work);
  for (std::thread& t : pool) t.join();
  long long total = 0;
  for (int i = 0; i < n; i++) {
    if (rc[i] < 0) return rc[i];
    total += res[i].iters;
  }
  return (int)std::min<long long>(total, 0x7fffffff);
}

// D^dag D (+ fmass^2) on device fields of many lattices in two launches
// (fermion_op_batch): the D of every lattice, then the D^dag of every
// lattice with the fmass^2 term.  Each lattice's intermediate field is its
// handle's DSq scratch field (allocated on the handle's first DSq).  The
// launches go to one stream, ordered after the work already queued on every
// handle's stream, and every handle's stream is ordered after them (events),
// so the call behaves like each handle's own DSq on its own stream.
namespace susy {
template <typename R>
FopArgs<R> batch_fop_args(susy_b200_lattice* h, const void* src, void* dst, const void* add,
                          double addc, double* dot, const int* skip) {
  typedef typename CT<R>::T T;
  const bool f64 = sizeof(R) == 8;
  FopArgs<R> a;
  a.g = h->g;
  a.U = (const T*)(f64 ? h->U : h->U32);
  a.Uinv = (const T*)(f64 ? h->Uinv : h->Uinv32);
  a.pd = (const T*)(f64 ? h->pd : h->pd32);
  a.src = (const T*)src;
  a.dst = (T*)dst;
  a.G = (R)h->G;
  a.doG = h->G > 1e-8;
  a.add = (const T*)add;
  a.addc = (R)addc;
  a.dot = dot;
  a.skip = skip;
  a.comp_major = 0;
  a.nsb = 0;
  a.nbrtab = h->nbrtab;
  a.eta_scale = (R)(h->rescale ? 2.0 : 1.0);
  a.trace = nullptr;
  return a;
}
template FopArgs<double> batch_fop_args<double>(susy_b200_lattice*, const void*, void*,
                                                const void*, double, double*, const int*);
template FopArgs<float> batch_fop_args<float>(susy_b200_lattice*, const void*, void*,
                                              const void*, double, double*, const int*);
}  // namespace susy

template <typename R>
static int dsq_batch(susy_b200_lattice* const* hs, const void* const* src, void* const* dst,
                     int n, cudaStream_t st) {
  const int prec = sizeof(R) == 8 ? 64 : 32;
  std::vector<void*> tmp(n);
  for (int i = 0; i < n; i++)
    if (!(tmp[i] = scratch_tf(hs[i], 0, prec))) return SUSY_B200_ENOMEM;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return SUSY_B200_ECUDA;
  }
  std::vector<cudaStream_t> others;
  for (int i = 0; i < n; i++)
    if (hs[i]->stream != st &&
        std::find(others.begin(), others.end(), hs[i]->stream) == others.end())
      others.push_back(hs[i]->stream);
  auto order = [](cudaStream_t from, cudaStream_t to) -> bool {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
    const bool ok = cudaEventRecord(e, from) == cudaSuccess && cudaStreamWaitEvent(to, e, 0) == cudaSuccess;
    cudaEventDestroy(e);   // released once the recorded work completes
    return ok;
  };
  for (cudaStream_t o : others)
    if (!order(o, st)) {
      cudaGetLastError();
      return SUSY_B200_ECUDA;
    }
  std::vector<FopArgs<R>> a(n);
  for (int i = 0; i < n; i++)
    a[i] = batch_fop_args<R>(hs[i], src[i], tmp[i], nullptr, 0.0, nullptr, nullptr);
  int rc = fermion_op_batch<R>(a.data(), n, hs[0]->N, 1, sms, st) < 0 ? SUSY_B200_EINVAL : 0;
  if (!rc) {
    for (int i = 0; i < n; i++) {
      const double fm = hs[i]->prm.fmass;
      const double fm2 = fm > 1e-8 ? fm * fm : 0.0;
      a[i] = batch_fop_args<R>(hs[i], tmp[i], dst[i], fm2 != 0.0 ? src[i] : nullptr, fm2,
                               nullptr, nullptr);
    }
    rc = fermion_op_batch<R>(a.data(), n, hs[0]->N, -1, sms, st) < 0 ? SUSY_B200_EINVAL : 0;
  }
  for (cudaStream_t o : others)
    if (!order(st, o) && !rc) rc = SUSY_B200_ECUDA;
  if (cudaGetLastError() != cudaSuccess && !rc) rc = SUSY_B200_ECUDA;
  return rc;
}

static_assert(FOP_BATCH_MAX == SUSY_B200_BATCH_MAX, "batch limit");

extern "C" int susy_b200_DSq_batch(susy_b200_lattice* const* hs, const void* const* src,
                                   void* const* dst, int n, int prec, void* cuda_stream) {
  if (!hs || !src || !dst || n < 1 || n > FOP_BATCH_MAX || (prec != 64 && prec != 32))
    return SUSY_B200_EINVAL;
  for (int i = 0; i < n; i++) {
    if (!hs[i] || !src[i] || !dst[i]) return SUSY_B200_EINVAL;
    if (hs[i]->N != hs[0]->N || hs[i]->prm.device != hs[0]->prm.device) return SUSY_B200_EINVAL;
  }
  if (cudaSetDevice(hs[0]->prm.device) != cudaSuccess) {
    cudaGetLastError();
    return SUSY_B200_ECUDA;
  }
  cudaStream_t st = cuda_stream ? (cudaStream_t)cuda_stream : hs[0]->stream;
  return prec == 64 ? dsq_batch<double>(hs, src, dst, n, st)
                    : dsq_batch<float>(hs, src, dst, n, st);
}

extern "C" int susy_b200_dev_congrad_multi_batch(susy_b200_lattice* const* hs,
                                                 const void* const* src,
                                                 void* const* const* psim, const int* norder,
                                                 const double* const* shift, int n, int MaxCG,
                                                 double errormin, double* size_r, int* iters,
                                                 void* cuda_stream) {
  if (!hs || !src || !psim || !norder || !shift || n < 1 || n > FOP_BATCH_MAX)
    return SUSY_B200_EINVAL;
  for (int i = 0; i < n; i++) {
    if (!hs[i] || !src[i] || !psim[i] || !shift[i] || norder[i] < 1 || norder[i] > MS_MAXS)
      return SUSY_B200_EINVAL;
    if (hs[i]->N != hs[0]->N || hs[i]->prm.device != hs[0]->prm.device) return SUSY_B200_EINVAL;
    for (int j = 0; j < norder[i]; j++)
      if (!psim[i][j]) return SUSY_B200_EINVAL;
    for (int k = 0; k < i; k++)
      if (hs[k] == hs[i]) return SUSY_B200_EINVAL;   // one solver state per handle
  }
  if (cudaSetDevice(hs[0]->prm.device) != cudaSuccess) {
    cudaGetLastError();
    return SUSY_B200_ECUDA;
  }
  cudaStream_t st = cuda_stream ? (cudaStream_t)cuda_stream : hs[0]->stream;
  const int rc = multishift_batch(hs, n, src, psim, norder, shift, MaxCG, errormin, size_r,
                                  iters, st);
  if (rc < 0) return rc;
  int most = 0;
  for (int i = 0; iters && i < n; i++) most = std::max(most, iters[i]);
  return most;
}
