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
