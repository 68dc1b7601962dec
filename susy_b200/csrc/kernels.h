// Host-side launch interface of the susy_b200 kernels (internal C++ API).
// All launches are asynchronous on the given stream; fields are in the
// device layout described in common.cuh.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace susy {

// Geometry from lattice extents, checked before anything is sized from it:
// even extents >= 2 (the reference's parity-ordered site layout,
// layout_hyper_prime.c:157-170, is a bijection only then), NCOL 2..4, PBC
// +-1, and the volume computed in 64 bits and bounded so that every 32-bit
// element index of one Twist_Fermion (16 NCOL^2 S complex) stays below
// INT_MAX.  Returns false (and leaves g untouched) otherwise.
bool make_geo(long nx, long ny, long nz, long nt, int ncol, int pbc, Geo* g);

constexpr int MS_MAXS = 32;
// Iterations per block of the blocked solution/search-vector update
constexpr int MS_BLK = 8;

// Device-resident state of one multi-shift solve (FP64 scalars)
struct MsState {
  double rsq, rsqstop, source_norm, cd;
  double rsqfreeze;   // shift j freezes once zeta_j^2 |r|^2 <= rsqfreeze (= rsqstop
                      // unless a caller stops the base system earlier)
  int iter, maxcg, nshift, skip, skip_b, pad;
  // blocked update: per-iteration coefficients of the current block
  // (hb = beta_j, 0 once shift j is frozen; hz = zeta_j(i+1); ha = alpha_j),
  // iterations recorded so far, iteration count at the block start, and
  // the shifts still live when the block began
  int record, blk_len, blk_start;
  unsigned done_r;    // blocks of the fused residual update finished so far
  int live[MS_MAXS];
  double hb[MS_BLK][MS_MAXS], hz[MS_BLK][MS_MAXS], ha[MS_BLK][MS_MAXS];
  double shift[MS_MAXS];
  double zeta_i[MS_MAXS], zeta_im1[MS_MAXS], zeta_ip1[MS_MAXS];
  double beta_i[MS_MAXS], beta_im1[MS_MAXS], alpha[MS_MAXS];
  int converged[MS_MAXS];   // 0 while shift j is live, else the iteration it froze at
  int active_p[MS_MAXS];
  // p_j update deferred to the next iteration's vector pass:
  // p_j <- pz_j r + pa_j p_j when pact_j
  double pz[MS_MAXS], pa[MS_MAXS];
  int pact[MS_MAXS];
};

struct MsVecs {
  void* p[MS_MAXS];    // p[0] = p0 (the DSq input), p[j] for shifts j >= 1
  void* psi[MS_MAXS];  // solutions
  void* r;
  void* mp;
};

// Vectors of the blocked solver: ring[i % (MS_BLK + 1)] holds the residual
// after i iterations; P[j] is shift j's search vector at the block start
// (P[0] a copy of the operator input p0 at that point); x[j] the solutions.
// p0_32 / mp32: FP32 operator input and output when the operator runs in
// FP32 (p0_32 written by the p0 update; nullptr in FP64).
// f32 = 1: ring and p0 are FP32 fields (the operator's input is p0 itself,
// its output mp32); the search vectors P and the solutions x stay FP64.
struct MsBlockVecs {
  void* ring[MS_BLK + 1];
  void* P[MS_MAXS];
  void* x[MS_MAXS];
  void* p0;
  void* mp;
  void* p0_32;
  void* mp32;
  int f32;
};

// fermion_op.cu, fermion_op_rows.cu
// Kernel variants: matrix per thread with the 16 output components
// interleaved block by block, the same with component-major block order,
// and one matrix row per thread (component-major).
// FOP_COMPACT evaluates all 220 products from a constant-memory term table;
// FOP_COMPACT_PF also prefetches the next product's operands.
// FOP_SITE_MAJOR_PP / FOP_COMP_MAJOR_PP: table-driven with two alternating
// operand buffers, site-major or component-major block order;
// FOP_SITE_MAJOR: site-major with one operand buffer (fewest registers);
// FOP_SITE_MAJOR_OCC / FOP_COMP_MAJOR_OCC: one buffer with the registers
// capped for 4 / 8 resident blocks of 128 threads per SM (128 / 64
// registers per thread): more resident warps to hide the L2 latency the
// operand gathers wait on, against a little spilling.  Measured at
// 12^3x24 U(3): the FP64 optimum is the 128-register site-major kernel
// (0.215 ms vs 0.260 uncapped; 102 registers: 0.256, 64: 0.59), the FP32 one
// the 64-register component-major kernel (0.117 ms vs 0.135; 48: 0.166).
// FOP_SITE_MAJOR_SHN / FOP_COMP_MAJOR_SHN: the _OCC kernels with each
// block's neighbour indices preloaded into shared memory.
// FOP_SITE_MAJOR_FRONT: site-major (FP64 4, FP32 8 blocks per SM) with the
// site component's long blocks at the front of the grid.
// FOP_GROUPED: one output component per warp over the same 32 sites, the
// components in groups of five that share operands (fermion_op_compact.cu;
// 3 resident blocks of 5 warps per SM in FP64, 6 in FP32).
// FOP_SITE_MAJOR_TR: FOP_SITE_MAJOR_FRONT after a pre-pass that writes
// every site's five determinant traces, which the site component's detLtoS
// term then reads instead of recomputing them at the site and its
// neighbours (needs the handle's 5 S complex trace field; without one it
// runs as FOP_SITE_MAJOR_FRONT).  The autotuner's pick in both precisions at
// 12^3x24 U(3).
enum { FOP_MAT = 0, FOP_MAT_CM = 1, FOP_ROWS = 2, FOP_COMPACT = 3, FOP_COMPACT_PF = 4,
       FOP_SITE_MAJOR_PP = 5, FOP_COMP_MAJOR_PP = 6, FOP_SITE_MAJOR = 7,
       FOP_SITE_MAJOR_OCC = 8, FOP_COMP_MAJOR_OCC = 9, FOP_SITE_MAJOR_SHN = 10,
       FOP_COMP_MAJOR_SHN = 11, FOP_SITE_MAJOR_FRONT = 12, FOP_GROUPED = 13,
       FOP_SITE_MAJOR_TR = 14, FOP_NVARIANTS = 15 };
template <typename R>
int fermion_op(const Geo& g, int N, const void* U, const void* Uinv, const void* pd,
                const void* src, void* dst, int sign, double G, const void* add, double addc,
                double* dot, const int* skip, int variant, const int* nbrtab, cudaStream_t st,
                double eta_scale = 1.0, void* trace = nullptr);
template <typename R> struct FopArgs;
template <typename R>
int fermion_op_rows(const FopArgs<R>& a, int N, int sign, cudaStream_t st);
int fop_partials(const Geo& g);
template <typename R>
int fermion_op_compact(const FopArgs<R>& a, int N, int sign, int variant, cudaStream_t st);
// One application over n <= FOP_BATCH_MAX lattices of one NCOL in a single
// persistent launch over a work table (fermion_op_compact.cu); the args
// carry no trace; a lattice's dot field receives 16 ceil(V / 128) partials.
// Returns the work items, < 0 on bad input.
constexpr int FOP_BATCH_MAX = 64;
template <typename R>
int fermion_op_batch(const FopArgs<R>* args, int n, int N, int sign, int sms, cudaStream_t st);
int upload_fop_terms(int device, cudaStream_t st);
int fop_ndisp();
void build_nbr_table(const Geo& g, int* tab, cudaStream_t st);

// derived.cu
void compute_uinv(const Geo& g, int N, const void* U, void* det, void* Uinv, cudaStream_t st);
void compute_plaqdet(const Geo& g, const void* det, void* pd, void* zw, cudaStream_t st);
void compute_dmuumu(const Geo& g, int N, const void* U, const void* pd, double G, void* D,
                    cudaStream_t st);
void compute_fmunu(const Geo& g, int N, const void* U, void* F, cudaStream_t st);

// layout.cu
void aos_to_soa(const Geo& g, int K, int N, const void* aos, void* soa, int prec, cudaStream_t st);
void soa_to_aos(const Geo& g, int K, int N, const void* soa, void* aos, int prec, cudaStream_t st);
void convert_field(long ncomplex, const void* in, int prec_in, void* out, int prec_out,
                   cudaStream_t st);

// cg.cu
int vec_blocks(long n);
void ms_init(MsState* st, const void* src, int prec, long n, double* part, int maxcg,
             double errormin, cudaStream_t s, int record = 0);
void ms_scalars1(MsState* st, const double* part, int np, cudaStream_t s);
void ms_scalars2(MsState* st, const double* part, int np, cudaStream_t s);
void ms_update_a(MsState* st, const MsVecs& v, int prec, int prec_x, long n, double* part,
                 cudaStream_t s);
int residual_partials(long n, const void* b, const void* ax, void* r64, void* r32, double* part,
                      cudaStream_t s);
void add_low(long n, const void* e32, void* x64, cudaStream_t s);
void scale_field(long n, double sc, void* x, cudaStream_t s);
void ms_update_b(MsState* st, const MsVecs& v, int prec, long n, cudaStream_t s);
void ms_update_fused(MsState* st, const MsVecs& v, int prec, int prec_x, long n, double* part,
                     cudaStream_t s);
void ms_update_p0(MsState* st, const MsVecs& v, int prec, long n, cudaStream_t s);
void norm2_partials(const void* x, int prec, long n, double* part, cudaStream_t s);
int rdot_partials(long n, const void* a, const void* b, double* part, cudaStream_t s);
void copy_field(long n, const void* a, void* b, cudaStream_t s);
// r(i) = r(i-1) + beta_0 mp, then (in the kernel's last block) the scalar
// recurrences of ms_scalars2 on |r(i)|^2
void msb_update_r(MsState* st, const MsBlockVecs& v, long n, double* part, bool mp32,
                  cudaStream_t s);
void msb_replace(MsState* st, const MsBlockVecs& v, long n, const void* rt, double rsq,
                 cudaStream_t s);
void msb_update_p0(MsState* st, const MsBlockVecs& v, long n, cudaStream_t s);
void msb_block(MsState* st, const MsBlockVecs& v, long n, cudaStream_t s);
void ms_set_stop(MsState* st, double errormin_base, cudaStream_t s);

// One lattice of a batched FP64 multi-shift solve (solver.cu): its state,
// vectors, field size, the operator's dot partials and the vector update's
// |r|^2 partials, and its blocks in the batch's table of vector blocks.
struct MsLat {
  MsState* st;
  MsVecs v;
  long n;          // complex entries of one Twist_Fermion
  double* part0;   // operator partials (16 ceil(V / 128) of them)
  int np0;
  double* part1;   // |r|^2 partials, one per vector block
  int vblk0;       // the lattice's first block in the batch's vector table
  int vblocks;     // its vector blocks, vec_blocks(n)
};
// The per-iteration kernels of ms_run for every lattice of a batch at once
// (L: a device array of nl MsLat; vtot: vector blocks of all lattices)
void ms_batch_scalars1(const MsLat* L, int nl, cudaStream_t s);
void ms_batch_update_fused(const MsLat* L, int nl, int vtot, cudaStream_t s);
void ms_batch_scalars2(const MsLat* L, int nl, cudaStream_t s);
void ms_batch_update_p0(const MsLat* L, int nl, int vtot, cudaStream_t s);
// out[i] = lattice i's stop flag
void ms_batch_skips(const MsLat* L, int nl, int* out, cudaStream_t s);

}  // namespace susy

namespace susy {
// force.cu
int force_blocks(const Geo& g);
int site_blocks(const Geo& g);
void fermion_force_pole(const Geo& g, int N, const void* U, const void* Uinv, const void* pd,
                        const void* sol, const void* psol, void* force, double amp, double G,
                        cudaStream_t st);
int mom_sub(long n, const void* force, void* mom, double eps, double* part, cudaStream_t st);
void axpy_field(long n, double s, const void* x, void* y, cudaStream_t st);
int gauge_force(const Geo& g, int N, const void* U, const void* Uinv, const void* pd,
                const void* zw, const void* D, const void* F, void* mom, double G, double bmass,
                double kappa, double kappa_u1, double eps, int det_only, double* part,
                cudaStream_t st);
int action_partials(const Geo& g, int N, const void* U, const void* D, const void* F,
                    const void* pd, const void* mom, double* part, cudaStream_t st);
int fermion_action_partials(long n, const void* src, int nsol, const void* const* sol_dev_array,
                            const double* amp_dev, double ampdeg, double* part, cudaStream_t st);
// rng.cu
void init_prn(const Geo& g, int seed, void* st, cudaStream_t s);
void gauss_fill(const Geo& g, int N, void* st, const void* gen, int K, int gen_outer, void* out,
                int* bad, cudaStream_t s);
}  // namespace susy
