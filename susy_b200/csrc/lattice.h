// Internal definition of the opaque handle declared in include/susy_b200.h.
#pragma once
#include <functional>
#include <vector>
#include "../../include/susy_b200.h"
#include "kernels.h"

namespace susy {
// Host copy of the reference's node generator (ranstuff.c:22-63)
struct HostPrn {
  uint32_t r[7], mult, add, ic;
};
}  // namespace susy

#define SUSY_NSCRATCH 8
#define SUSY_NPART 4

struct susy_b200_lattice {
  susy_b200_params prm;
  susy::Geo g;
  int N = 2;
  double G = 0.0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  // FP64 lattice fields (device layout, common.cuh)
  void *U = nullptr, *mom = nullptr, *Uinv = nullptr, *force = nullptr;
  void *det = nullptr, *pd = nullptr, *zw = nullptr, *D = nullptr, *F = nullptr;
  // FP32 copies read by the FP32 operator
  void *U32 = nullptr, *Uinv32 = nullptr, *pd32 = nullptr;
  void* stage = nullptr;  // AoS staging buffer (one FP64 Twist_Fermion)
  int* nbrtab = nullptr;  // neighbour index table of the table-driven operator
  void* trace[2] = {};    // determinant traces of FOP_SITE_MAJOR_TR (FP64, FP32);
                          // each solver context owns its own
  susy::MsState* ms = nullptr;
  void* tf64[SUSY_NSCRATCH] = {};
  void* tf32[SUSY_NSCRATCH] = {};
  double* part[SUSY_NPART] = {};
  std::vector<void*> sols;    // solutions for the host-facing CG
  std::vector<void*> pvec64;  // p_j of the FP64 multi-shift CG
  std::vector<void*> pvec32;
  std::vector<void*> ring;    // residual ring of the blocked FP64 solver
  std::vector<void*> vec32;   // FP32 residual ring of the mixed solver's FP32 phase
  int mix_vec32 = 0;          // mixed solver: FP32 residuals and p0 in its FP32 phase
  int rescale = 0;            // the reference's RESCALE: eta doubled in and out of fermion_op
  double* meas = nullptr;     // measurement partials
  size_t meas_n = 0;
  int ms_blocked = 1;         // FP64 multi-shift CG: blocked vector update
  int use_graphs = 1;         // replay the solver's iteration chunks as CUDA graphs
  int host_solver = 0;        // solver behind susy_b200_congrad_multi
  double mix_switch = 3e-4;   // mixed solver: FP32 operator once |r| < this |src|
  double mix_reliable = 1e-2; // mixed solver: true residual when |r| fell this much
  int mix_interval = 0;       // mixed solver: > 0, true residual every this many iterations
  int mix_correct32 = 1;      // mixed solver: per-shift corrections with the FP32 operator
  std::vector<void*> extra;   // other lazily allocated fields
  int* poll = nullptr;        // pinned host words for solver polling
  // trajectory state (hmc.cu)
  double* bigpart = nullptr;
  long bigpart_n = 0;
  void* gen = nullptr;        // U(N) generators
  void* prn = nullptr;        // per-site generator states
  int* rng_bad = nullptr;
  void* ptrbuf = nullptr;     // device copy of field pointers / coefficients
  std::vector<void*> gsrc, gr_psim, traj_psim, extra5, refine;
  susy::HostPrn node_prn = {};
  // second solver context (hmc.cu solve_pfs): its own stream, solver state
  // and scratch; the links, derived fields and neighbour table are this
  // handle's (shares_fields set in the context)
  susy_b200_lattice* shadow = nullptr;
  bool shares_fields = false;
  int pf_streams = 1;         // overlap the pseudofermion solves of a trajectory
  cudaStream_t copy = nullptr;   // host congrad_multi: early solution copies
  cudaEvent_t copy_ev = nullptr;
  int fop_variant[2] = {-1, -1};  // chosen operator kernel (FP64, FP32); -1 = tune
  float fop_ms[2][SUSY_B200_FOP_NVARIANTS] = {};  // autotuner timings per variant
  int err = 0, cuda_err = 0;
};

namespace susy {
bool ck(susy_b200_lattice* h, cudaError_t e);
int set_err(susy_b200_lattice* h, int code);
void* dalloc(susy_b200_lattice* h, size_t bytes);
size_t field_bytes(const susy_b200_lattice* h, int K, int prec);
int upload_links(susy_b200_lattice* h, void* dev, const double* host, size_t stride, int K);
int download_links(susy_b200_lattice* h, const void* dev, double* host, size_t stride, int K);
int refresh_derived(susy_b200_lattice* h);
void refresh_low(susy_b200_lattice* h);
int dev_fop(susy_b200_lattice* h, const void* src, void* dst, int sign, int prec,
            const void* add, double addc, double* dot, const int* skip);
int autotune_fop(susy_b200_lattice* h, int prec);
void* scratch_tf(susy_b200_lattice* h, int which, int prec);
double* partials(susy_b200_lattice* h, int which);
long tf_complex(const susy_b200_lattice* h);
void* sol_field(susy_b200_lattice* h, int j);
susy_b200_lattice* solver_shadow(susy_b200_lattice* h);
cudaStream_t copy_stream(susy_b200_lattice* h);
// Called by the blocked solver at a poll for each shift j >= 1 whose
// solution the multi-shift pass has finished (the shift froze and its last
// block pass ran): the host API copies it out while the solve goes on
typedef std::function<void(int)> FrozenHook;
int multishift_fp64(susy_b200_lattice* h, const void* src, void* const* psim, int norder,
                    const double* shift, int MaxCG, double errormin, double* size_r,
                    int* iters, const FrozenHook* on_frozen = nullptr);
int measure(susy_b200_lattice* h, susy_b200_meas* m);
int multishift_batch(susy_b200_lattice* const* hs, int nl, const void* const* src,
                     void* const* const* psim, const int* norder, const double* const* shift,
                     int MaxCG, double errormin, double* size_r, int* iters, cudaStream_t st);
// The operator arguments of lattice h for the batched operator
// (fermion_op_batch): its geometry, fields of precision R, couplings,
// neighbour table and RESCALE factor (batch.cu)
template <typename R>
FopArgs<R> batch_fop_args(susy_b200_lattice* h, const void* src, void* dst, const void* add,
                          double addc, double* dot, const int* skip);
int net_apply(susy_b200_net* n, const void* src, void* dst);
int multishift_learned(susy_b200_lattice* h, susy_b200_net* net, const void* src,
                       void* const* psim, int norder, const double* shift, int MaxCG,
                       double errormin, int nrefine, double loose, double* size_r, int* iters,
                       int* refine_iters);
}  // namespace susy
