// Table-driven variant of the fermion operator (same terms as
// fermion_op.cu, 4d_Q16/susy/utilities.c:141-865).
//
// Every one of the 160 distinct NCOL x NCOL products per site (the 220 of
// the reference with its coinciding PtoP pairs merged, fop_table.cuh) is one
// row of a term table in constant memory (coefficient, temporal-BC
// displacement, and the component and neighbour displacement of each
// factor), grouped by operand pattern so that which fields enter and which
// are adjointed is known at compile time.  Neighbour indices come from a
// per-lattice table (tab[d * S + s], one coalesced int per factor) instead
// of per-term wrap arithmetic.  A thread loops over the 10 terms of its
// output matrix,
// optionally with the next term's operands prefetched.  The loop bodies are
// a few hundred instructions, so the instruction working set stays in the
// SM's instruction cache (the fully unrolled kernels stall on instruction
// fetch) and only one or two products' operands are live.  The determinant
// terms (detStoL, detLtoS, G != 0) follow the loops.
#include <algorithm>
#include <mutex>
#include <vector>
#include "common.cuh"
#include "fop.cuh"
#include "fop_table.cuh"
#include "kernels.h"

namespace susy {

__constant__ FTerm c_terms[MAX_TERMS];
__constant__ short c_pat_start[NTF][NPAT + 1];
__constant__ char4 c_disp[MAX_DISP];
// Distinct displacements of each output component's products (at most 10):
// the blocks of the shared-index kernels preload those neighbour indices
// into shared memory; FTerm.sl / .sr are a product's slots in that list.
constexpr int MAX_SLOTS = 12;
__constant__ int8_t c_slot_disp[NTF][MAX_SLOTS];
__constant__ int8_t c_nslot[NTF];

const TermBuilder& fop_terms() {
  static const TermBuilder tb = [] {
    TermBuilder b;
    b.build();
    return b;
  }();
  return tb;
}

template <typename R>
static void prefer_l1_grouped();

static std::mutex g_terms_mu;
static bool g_terms_ready[64];

int upload_fop_terms(int device, cudaStream_t st) {
  (void)st;
  std::lock_guard<std::mutex> lk(g_terms_mu);
  if (device >= 0 && device < 64 && g_terms_ready[device]) return 0;
  const TermBuilder& tb = fop_terms();
  std::vector<FTerm> flat;
  short start[NTF][NPAT + 1];
  int8_t slot_disp[NTF][MAX_SLOTS] = {};
  int8_t nslot[NTF] = {};
  auto slot = [&](int c, int d) -> int {
    for (int j = 0; j < nslot[c]; j++)
      if (slot_disp[c][j] == d) return j;
    if (nslot[c] >= MAX_SLOTS) return -1;
    slot_disp[c][nslot[c]] = (int8_t)d;
    return nslot[c]++;
  };
  for (int c = 0; c < NTF; c++)
    for (int p = 0; p < NPAT; p++) {
      start[c][p] = (short)flat.size();
      for (FTerm T : tb.terms[c][p]) {
        const int a = slot(c, T.dl), b = slot(c, T.dr);
        if (a < 0 || b < 0) return -1;
        T.sl = (int8_t)a;
        T.sr = (int8_t)b;
        flat.push_back(T);
      }
      start[c][p + 1] = (short)flat.size();
    }
  if ((int)flat.size() > MAX_TERMS || (int)tb.disp.size() > MAX_DISP) return -1;
  cudaMemcpyToSymbol(c_terms, flat.data(), flat.size() * sizeof(FTerm));
  cudaMemcpyToSymbol(c_pat_start, start, sizeof(start));
  cudaMemcpyToSymbol(c_disp, tb.disp.data(), tb.disp.size() * sizeof(char4));
  cudaMemcpyToSymbol(c_slot_disp, slot_disp, sizeof(slot_disp));
  cudaMemcpyToSymbol(c_nslot, nslot, sizeof(nslot));
  if (cudaGetLastError() != cudaSuccess) return -2;
  prefer_l1_grouped<double>();
  prefer_l1_grouped<float>();
  if (device >= 0 && device < 64) g_terms_ready[device] = true;
  return 0;
}

int fop_ndisp() { return (int)fop_terms().disp.size(); }

// Neighbour index table: tab[d * S + s] = index of s + disp[d]
__global__ void k_nbr_table(Geo g, int nd, int* tab) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const Site c = site_of(g, s);
  for (int d = 0; d < nd; d++) {
    const char4 v = c_disp[d];
    tab[(size_t)d * g.S + s] = nbr(g, c, v.x, v.y, v.z, v.w);
  }
}

void build_nbr_table(const Geo& g, int* tab, cudaStream_t st) {
  count_launch(), k_nbr_table<<<(g.V + 127) / 128, 128, 0, st>>>(g, fop_ndisp(), tab);
}

// ---------------------------------------------------------------------------
// Device
// One pattern's terms: compile-time operand fields and adjoints
template <int N, typename R, int SIGN, int PAT, bool PF>
SUSY_D void run_pattern(Mat<N, R>& acc, const FopArgs<R>& a, int s, unsigned bcm, int t0,
                        int t1) {
  constexpr bool LF = (PAT == P_FU || PAT == P_FUD);         // left factor is the source
  constexpr bool RF = !LF;
  constexpr bool AL = (PAT == P_UDF) ^ (LF && SIGN < 0);
  constexpr bool AR = (PAT == P_FUD) ^ (RF && SIGN < 0);
  const int S = a.g.S;
  const typename CT<R>::T* fl = LF ? a.src : a.U;
  const typename CT<R>::T* fr = RF ? a.src : a.U;
  const R pbc = (R)a.g.pbc;
  if (t0 >= t1) return;
  if (PF) {
    FTerm T = c_terms[t0];
    Mat<N, R> L = ldm<N, R, AL>(fl, T.kl, a.nbrtab[(size_t)T.dl * S + s], S);
    Mat<N, R> Rm = ldm<N, R, AR>(fr, T.kr, a.nbrtab[(size_t)T.dr * S + s], S);
#pragma unroll 1
    for (int t = t0; t < t1; t++) {
      Mat<N, R> Ln, Rn;
      FTerm Tn = T;
      if (t + 1 < t1) {
        Tn = c_terms[t + 1];
        Ln = ldm<N, R, AL>(fl, Tn.kl, a.nbrtab[(size_t)Tn.dl * S + s], S);
        Rn = ldm<N, R, AR>(fr, Tn.kr, a.nbrtab[(size_t)Tn.dr * S + s], S);
      }
      mac<0>(acc, (R)T.coef * bc_of<R>(bcm, T.bcdt, pbc) * ((LF ? T.kl : T.kr) ? (R)1 : a.eta_scale),
             L, Rm);
      L = Ln;
      Rm = Rn;
      T = Tn;
    }
  } else {
#pragma unroll 1
    for (int t = t0; t < t1; t++) {
      const FTerm T = c_terms[t];
      Mat<N, R> L = ldm<N, R, AL>(fl, T.kl, a.nbrtab[(size_t)T.dl * S + s], S);
      Mat<N, R> Rm = ldm<N, R, AR>(fr, T.kr, a.nbrtab[(size_t)T.dr * S + s], S);
      mac<0>(acc, (R)T.coef * bc_of<R>(bcm, T.bcdt, pbc) * ((LF ? T.kl : T.kr) ? (R)1 : a.eta_scale),
             L, Rm);
    }
  }
}

constexpr int CT_THREADS = 128;

template <int N, typename R, int SIGN, bool PREFETCH>
__global__ void __launch_bounds__(CT_THREADS)
fermion_op_compact_kernel(FopArgs<R> a) {
  if (a.skip && *a.skip) return;
  const int comp = blockIdx.x / a.nsb;
  const int s = (blockIdx.x % a.nsb) * CT_THREADS + threadIdx.x;
  double part = 0.0;
  if (s < a.g.V) {
    const Site c = site_of(a.g, s);
    const unsigned bcm = bc_mask(a.g, c);
    Mat<N, R> acc;
    acc.zero();
    run_pattern<N, R, SIGN, P_UF, PREFETCH>(acc, a, s, bcm, c_pat_start[comp][0],
                                             c_pat_start[comp][1]);
    run_pattern<N, R, SIGN, P_FU, PREFETCH>(acc, a, s, bcm, c_pat_start[comp][1],
                                             c_pat_start[comp][2]);
    run_pattern<N, R, SIGN, P_FUD, PREFETCH>(acc, a, s, bcm, c_pat_start[comp][2],
                                              c_pat_start[comp][3]);
    run_pattern<N, R, SIGN, P_UDF, PREFETCH>(acc, a, s, bcm, c_pat_start[comp][3],
                                              c_pat_start[comp][4]);
    if (a.doG) {
      if (comp == 0)
        det_ltos_rt<N, R, SIGN>(acc, a, c);
      else if (comp <= NUMLINK)
        det_stol_rt<N, R, SIGN>(acc, a, c, comp - 1);
    }
    if (comp == 0) eta_rescale(acc, a.eta_scale);
    if (SIGN < 0) {
      Mat<N, R> t = acc;
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) acc.e[i][j] = Cx<R>(-t.e[j][i].re, t.e[j][i].im);
    }
    if (a.add) {
      Mat<N, R> x = ldm<N, R>(a.add, comp, s, a.g.S);
      axpy(acc, Cx<R>(a.addc, 0), x);
      if (a.dot) part = rdot(x, acc);
    }
    stm<N, R>(a.dst, comp, s, a.g.S, acc);
  }
  if (a.dot) {
    part = block_sum<CT_THREADS>(part);
    if (threadIdx.x == 0) a.dot[blockIdx.x] = part;
  }
}

// ---------------------------------------------------------------------------
// Second generation of the table-driven kernels.
//
// Site-major block order: the 16 blocks of one site tile (one per output
// component) are adjacent in the grid, so they run at the same time and
// the tile's neighbourhood (source, links, U^-1, plaquette determinants
// within three steps) is fetched from HBM once and then served from L2 to
// all 16; with component-major order every output component sweeps the
// whole lattice and the links are re-read from HBM per component.
//
// Two operand buffers used alternately: the next product's operands are in
// flight while the current one is multiplied, with no register copies
// between iterations (a rolled loop with one prefetch buffer copies both
// matrices every term).  Both block orders are built; which one wins
// depends on the precision (the autotuner decides).

// PP = false: one operand buffer, no prefetch (fewest registers).
// shn != nullptr: neighbour indices from the block's shared-memory copy
// (shn[slot * CT_THREADS + threadIdx.x]) instead of the global table.
template <int N, typename R, int SIGN, int PAT, bool PP, typename ACC>
SUSY_D void run_pattern_pp(ACC& acc, const FopArgs<R>& a, int s, unsigned bcm, int t0, int t1,
                           const int* shn = nullptr) {
  constexpr bool LF = (PAT == P_FU || PAT == P_FUD);
  constexpr bool RF = !LF;
  constexpr bool AL = (PAT == P_UDF) ^ (LF && SIGN < 0);
  constexpr bool AR = (PAT == P_FUD) ^ (RF && SIGN < 0);
  const int S = a.g.S;
  const typename CT<R>::T* fl = LF ? a.src : a.U;
  const typename CT<R>::T* fr = RF ? a.src : a.U;
  const R pbc = (R)a.g.pbc;
  if (t0 >= t1) return;
  if (!PP) {
#pragma unroll 1
    for (int t = t0; t < t1; t++) {
      const FTerm T = c_terms[t];
      const int il = shn ? shn[T.sl * CT_THREADS + threadIdx.x] : a.nbrtab[(size_t)T.dl * S + s];
      const int ir = shn ? shn[T.sr * CT_THREADS + threadIdx.x] : a.nbrtab[(size_t)T.dr * S + s];
      const Mat<N, R> L = ldm<N, R, AL>(fl, T.kl, il, S);
      const Mat<N, R> Rm = ldm<N, R, AR>(fr, T.kr, ir, S);
      acc.add((R)T.coef * bc_of<R>(bcm, T.bcdt, pbc) * ((LF ? T.kl : T.kr) ? (R)1 : a.eta_scale), L, Rm);
    }
    return;
  }
  FTerm TA = c_terms[t0];
  Mat<N, R> LA = ldm<N, R, AL>(fl, TA.kl, a.nbrtab[(size_t)TA.dl * S + s], S);
  Mat<N, R> RA = ldm<N, R, AR>(fr, TA.kr, a.nbrtab[(size_t)TA.dr * S + s], S);
#pragma unroll 1
  for (int t = t0;; t += 2) {
    FTerm TB;
    Mat<N, R> LB, RB;
    const bool hb = t + 1 < t1;
    if (hb) {
      TB = c_terms[t + 1];
      LB = ldm<N, R, AL>(fl, TB.kl, a.nbrtab[(size_t)TB.dl * S + s], S);
      RB = ldm<N, R, AR>(fr, TB.kr, a.nbrtab[(size_t)TB.dr * S + s], S);
    }
    acc.add((R)TA.coef * bc_of<R>(bcm, TA.bcdt, pbc) * ((LF ? TA.kl : TA.kr) ? (R)1 : a.eta_scale),
              LA, RA);
    if (!hb) break;
    const bool ha = t + 2 < t1;
    if (ha) {
      TA = c_terms[t + 2];
      LA = ldm<N, R, AL>(fl, TA.kl, a.nbrtab[(size_t)TA.dl * S + s], S);
      RA = ldm<N, R, AR>(fr, TA.kr, a.nbrtab[(size_t)TA.dr * S + s], S);
    }
    acc.add((R)TB.coef * bc_of<R>(bcm, TB.bcdt, pbc) * ((LF ? TB.kl : TB.kr) ? (R)1 : a.eta_scale),
              LB, RB);
    if (!ha) break;
  }
}

// Longest blocks first.  The site component's blocks cost ~3.5x the others
// (its determinant epilogue, det_ltos_rt, loads 470 complex numbers against
// 180 for ten products).  Block b of a grid of 16 blocks per tile over
// ntile tiles: the ntile site-component blocks first, then the other 15
// blocks of each tile, tile by tile.  Returns the tile, and k = 0 for the
// site component, 1..15 for the others.  Measured at 12^3x24 U(3) on one
// box: the site-major kernel in this order 0.171 ms (FP64) and 0.0996 ms
// (FP32) per launch against 0.191 and 0.129 with every tile's 16 blocks
// adjacent (and 0.107 for the component-major FP32 kernel).  The price is
// DRAM traffic in FP64, whose fields exceed L2: the site-component sweep
// and the sweep of the other 15 each stream the lattice, 372 MB per launch
// against 288 MB (264 MB algorithmic); in FP32 141 MB (132 algorithmic).
// Super-chunks of 48 tiles, each with its site-component blocks first,
// kept the traffic down but not the time (FP64 0.189 ms).
SUSY_D int front_block(int b, int ntile, int& k) {
  if (b < ntile) {
    k = 0;
    return b;
  }
  b -= ntile;
  k = 1 + b % 15;
  return b / 15;
}

// Block order: site-major (SM = true) or component-major; PP: two operand
// buffers (prefetch) or one.
// SHN: the block first copies its output component's neighbour indices
// (at most MAX_SLOTS displacements x CT_THREADS sites) into shared memory,
// so a product's operand loads no longer wait on a global index load.
// FRONT (with SM): the site component's blocks first, then the others
// site-major (front_block).  TR: detLtoS from the pre-pass's traces.
template <int N, typename R, int SIGN, bool SM, bool PP, int MINB, bool SHN = false,
          bool FRONT = false, bool TR = false>
__global__ void __launch_bounds__(CT_THREADS, MINB)
fermion_op_pp_kernel(FopArgs<R> a) {
  if (a.skip && *a.skip) return;
  int comp, tile;
  if (FRONT) {
    tile = front_block(blockIdx.x, a.nsb, comp);
  } else {
    comp = SM ? blockIdx.x % NTF : blockIdx.x / a.nsb;
    tile = SM ? blockIdx.x / NTF : blockIdx.x % a.nsb;
  }
  const int s = tile * CT_THREADS + threadIdx.x;
  __shared__ int shn[SHN ? MAX_SLOTS * CT_THREADS : 1];
  if (SHN) {
    const int ns = c_nslot[comp];
    for (int j = 0; j < ns; j++)
      shn[j * CT_THREADS + threadIdx.x] =
          s < a.g.V ? a.nbrtab[(size_t)c_slot_disp[comp][j] * a.g.S + s] : 0;
    __syncthreads();
  }
  const int* sh = SHN ? shn : nullptr;
  double part = 0.0;
  if (s < a.g.V) {
    const Site c = site_of(a.g, s);
    const unsigned bcm = bc_mask(a.g, c);
    AccMat<N, R> acc;
    acc.zero();
    run_pattern_pp<N, R, SIGN, P_UF, PP>(acc, a, s, bcm, c_pat_start[comp][0], c_pat_start[comp][1], sh);
    run_pattern_pp<N, R, SIGN, P_FU, PP>(acc, a, s, bcm, c_pat_start[comp][1], c_pat_start[comp][2], sh);
    run_pattern_pp<N, R, SIGN, P_FUD, PP>(acc, a, s, bcm, c_pat_start[comp][2], c_pat_start[comp][3], sh);
    run_pattern_pp<N, R, SIGN, P_UDF, PP>(acc, a, s, bcm, c_pat_start[comp][3], c_pat_start[comp][4], sh);
    Mat<N, R> out = acc.get();
    part = fop_finish<N, R, SIGN, TR>(out, a, c, comp);
  }
  if (a.dot) {
    part = block_sum<CT_THREADS>(part);
    if (threadIdx.x == 0) a.dot[blockIdx.x] = part;
  }
}

// Grouped block shape: output components that read the same operands run
// in one block, one warp each, over the same 32 sites, so an operand one
// warp fetched is still in the SM's L1 when the next warp of the block asks
// for it.  Counted over the 160 products, the 15 link and plaquette
// components read 295 (field, component, displacement) operands per site
// when each is fetched on its own; in three groups of five -- psi'_0..4,
// chi'_01..chi'_12, chi'_13..chi'_34 (component order) -- they read 211
// (e.g. chi_eB(x) is read by both psi'_e and psi'_B, U_e(x - e) by every
// psi'_B; a search over swaps between groups finds no split into fives
// that reads fewer).  The site component, whose determinant epilogue
// (detLtoS) costs ~3.5x its products, runs in blocks of its own (5 warps
// over 160 sites), so no block waits on one slow warp.  A chunk of 160
// sites has one site-component block and the 15 group blocks of its five
// 32-site tiles, in front_block's order.
// Measured at 12^3x24 U(3) (ncu): the L1 hit rate rises from 6-9% to 30%
// and the L2 -> L1 traffic falls by 25% (FP64 2.30 -> 1.72 GB, FP32 1.17 ->
// 0.88 GB per launch), yet the kernel is no faster than the site-major one
// (FP64 0.205 against 0.171 ms, FP32 0.109 against 0.100): with 15
// resident warps per SM of which few have a load in flight, the operand
// gathers are bound by latency, not by L2 bandwidth.  With each chunk's 16
// blocks adjacent instead, DRAM traffic fell from 365 to 281 MB (FP64) but
// the kernel took 0.239 / 0.154 ms; blocks of 15 warps (all 15 components,
// 161 operands per site): 0.224 / 0.117 ms.
constexpr int GRP_WARPS = 5;
constexpr int GRP_THREADS = 32 * GRP_WARPS;

template <int N, typename R, int SIGN, int MINB>
__global__ void __launch_bounds__(GRP_THREADS, MINB)
fermion_op_grp_kernel(FopArgs<R> a) {
  if (a.skip && *a.skip) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int k;
  const int chunk = front_block(blockIdx.x, a.nsb, k);
  int comp, s;
  if (k == 0) {
    comp = 0;
    s = chunk * GRP_THREADS + threadIdx.x;
  } else {
    comp = 1 + ((k - 1) % 3) * GRP_WARPS + warp;
    s = (chunk * GRP_WARPS + (k - 1) / 3) * 32 + lane;
  }
  double part = 0.0;
  if (s < a.g.V) {
    const Site c = site_of(a.g, s);
    const unsigned bcm = bc_mask(a.g, c);
    AccMat<N, R> acc;
    acc.zero();
    run_pattern_pp<N, R, SIGN, P_UF, false>(acc, a, s, bcm, c_pat_start[comp][0], c_pat_start[comp][1]);
    run_pattern_pp<N, R, SIGN, P_FU, false>(acc, a, s, bcm, c_pat_start[comp][1], c_pat_start[comp][2]);
    run_pattern_pp<N, R, SIGN, P_FUD, false>(acc, a, s, bcm, c_pat_start[comp][2], c_pat_start[comp][3]);
    run_pattern_pp<N, R, SIGN, P_UDF, false>(acc, a, s, bcm, c_pat_start[comp][3], c_pat_start[comp][4]);
    Mat<N, R> out = acc.get();
    part = fop_finish<N, R, SIGN>(out, a, c, comp);
  }
  if (a.dot) {
    part = block_sum<GRP_THREADS>(part);
    if (threadIdx.x == 0) a.dot[blockIdx.x] = part;
  }
}

// Blocks: 16 per 160-site chunk, 16 ceil(V / 160) in all, within the
// 16 ceil(V / 32) dot partials fop_partials() sizes.  Resident blocks per
// SM: 3 in FP64 (at most 136 registers a thread), 6 in FP32 (68).
template <int N, typename R>
static int launch_grp(FopArgs<R> a, int sign, cudaStream_t st) {
  constexpr int MINB = sizeof(R) == 8 ? 3 : 6;
  a.nsb = (a.g.V + GRP_THREADS - 1) / GRP_THREADS;
  const int nblk = 16 * a.nsb;
  if (sign > 0)
    count_launch(), fermion_op_grp_kernel<N, R, 1, MINB><<<nblk, GRP_THREADS, 0, st>>>(a);
  else
    count_launch(), fermion_op_grp_kernel<N, R, -1, MINB><<<nblk, GRP_THREADS, 0, st>>>(a);
  return nblk;
}

// The grouped kernels use 40 B of shared memory: ask for the largest L1
// split, the cache the grouping relies on.  A preference of the current
// device, set with the term table at lattice creation (outside any stream
// capture); a refusal only costs speed.
template <typename R>
static void prefer_l1_grouped() {
  constexpr int MINB = sizeof(R) == 8 ? 3 : 6;
  const void* k[6] = {(const void*)fermion_op_grp_kernel<2, R, 1, MINB>,
                      (const void*)fermion_op_grp_kernel<2, R, -1, MINB>,
                      (const void*)fermion_op_grp_kernel<3, R, 1, MINB>,
                      (const void*)fermion_op_grp_kernel<3, R, -1, MINB>,
                      (const void*)fermion_op_grp_kernel<4, R, 1, MINB>,
                      (const void*)fermion_op_grp_kernel<4, R, -1, MINB>};
  for (const void* f : k)
    if (cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 0) != cudaSuccess)
      cudaGetLastError();
}

template <int N, typename R, bool PF>
static int launch_compact(FopArgs<R> a, int sign, cudaStream_t st) {
  a.nsb = (a.g.V + CT_THREADS - 1) / CT_THREADS;
  const int nblk = a.nsb * NTF;
  if (sign > 0)
    count_launch(), fermion_op_compact_kernel<N, R, 1, PF><<<nblk, CT_THREADS, 0, st>>>(a);
  else
    count_launch(), fermion_op_compact_kernel<N, R, -1, PF><<<nblk, CT_THREADS, 0, st>>>(a);
  return nblk;
}

template <int N, typename R, bool SM, bool PP, int MINB = 1, bool SHN = false, bool FRONT = false,
          bool TR = false>
static int launch_pp(FopArgs<R> a, int sign, cudaStream_t st) {
  a.nsb = (a.g.V + CT_THREADS - 1) / CT_THREADS;
  const int nblk = a.nsb * NTF;
  if (TR && a.doG) {   // the traces detLtoS reads, for this sign's source
    const dim3 nb((a.g.V + CT_THREADS - 1) / CT_THREADS, NUMLINK);
    if (sign > 0)
      count_launch(), k_det_traces<N, R, false><<<nb, CT_THREADS, 0, st>>>(a);
    else
      count_launch(), k_det_traces<N, R, true><<<nb, CT_THREADS, 0, st>>>(a);
  }
  if (sign > 0)
    count_launch(), fermion_op_pp_kernel<N, R, 1, SM, PP, MINB, SHN, FRONT, TR><<<nblk, CT_THREADS, 0, st>>>(a);
  else
    count_launch(), fermion_op_pp_kernel<N, R, -1, SM, PP, MINB, SHN, FRONT, TR><<<nblk, CT_THREADS, 0, st>>>(a);
  return nblk;
}

// ---------------------------------------------------------------------------
// One operator application over many independent lattices of one NCOL in a
// single persistent launch (susy_b200_DSq_batch).  The work table is the
// site-major order of the table-driven kernels with every site-component
// item first (front_block's reason, across the whole batch): item w < T,
// T = the lattices' 128-site tiles in all, is the site-component block of
// global tile w; item T + q is output component 1 + q % 15 of global tile
// q / 15; a global tile belongs to the lattice whose tile range holds it.
// Each lattice keeps its own geometry, fields, couplings and neighbour
// table (FopArgs), all passed in the kernel's parameter space, so the
// launch needs no device memory of its own.  The grid is resident-sized
// (blocks per SM x SMs) and every block walks the table with a stride of
// the grid, so lattices of 256 sites and of 8192 fill the GPU together.
// The products, determinant terms and epilogue are those of
// fermion_op_pp_kernel (one operand buffer), so each lattice gets the same
// result as its own site-major launch.  A lattice whose skip flag is set
// (its solve has finished) contributes no work; with a dot field, lattice
// i's item (tile t, component k) writes its block's share of the epilogue's
// inner product to dot[k * tiles_i + t] (16 tiles_i partials per lattice).
template <typename R>
struct FopBatch {
  int n;                          // lattices
  int tiles;                      // T: 128-site tiles of all lattices
  int start[FOP_BATCH_MAX + 1];   // first global tile of lattice i
  FopArgs<R> a[FOP_BATCH_MAX];
};
// kernel parameters may take up to 32764 bytes (CUDA 12.1 and later)
static_assert(sizeof(FopBatch<double>) <= 32000, "batch arguments exceed the parameter space");

// Largest i < n with start[i] <= t
SUSY_D int batch_lattice(const int* start, int n, int t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= t)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <int N, typename R, int SIGN, int MINB>
__global__ void __launch_bounds__(CT_THREADS, MINB)
fermion_op_batch_kernel(const __grid_constant__ FopBatch<R> B) {
  const int total = 16 * B.tiles;
#pragma unroll 1
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    int gt, comp;
    if (w < B.tiles) {
      gt = w;
      comp = 0;
    } else {
      gt = (w - B.tiles) / 15;
      comp = 1 + (w - B.tiles) % 15;
    }
    const int i = batch_lattice(B.start, B.n, gt);
    const FopArgs<R>& a = B.a[i];
    if (a.skip && *a.skip) continue;   // the whole block: one lattice per item
    const int tile = gt - B.start[i];
    const int s = tile * CT_THREADS + threadIdx.x;
    double part = 0.0;
    if (s < a.g.V) {
      const Site c = site_of(a.g, s);
      const unsigned bcm = bc_mask(a.g, c);
      AccMat<N, R> acc;
      acc.zero();
      run_pattern_pp<N, R, SIGN, P_UF, false>(acc, a, s, bcm, c_pat_start[comp][0], c_pat_start[comp][1]);
      run_pattern_pp<N, R, SIGN, P_FU, false>(acc, a, s, bcm, c_pat_start[comp][1], c_pat_start[comp][2]);
      run_pattern_pp<N, R, SIGN, P_FUD, false>(acc, a, s, bcm, c_pat_start[comp][2], c_pat_start[comp][3]);
      run_pattern_pp<N, R, SIGN, P_UDF, false>(acc, a, s, bcm, c_pat_start[comp][3], c_pat_start[comp][4]);
      Mat<N, R> out = acc.get();
      part = fop_finish<N, R, SIGN>(out, a, c, comp);
    }
    if (a.dot) {
      part = block_sum<CT_THREADS>(part);
      if (threadIdx.x == 0) a.dot[comp * (B.start[i + 1] - B.start[i]) + tile] = part;
      __syncthreads();   // block_sum's shared words are reused by the next item
    }
  }
}

template <int N, typename R>
static void launch_batch(const FopBatch<R>& B, int sign, int grid, cudaStream_t st) {
  constexpr int MINB = sizeof(R) == 8 ? 4 : 8;
  if (sign > 0)
    count_launch(), fermion_op_batch_kernel<N, R, 1, MINB><<<grid, CT_THREADS, 0, st>>>(B);
  else
    count_launch(), fermion_op_batch_kernel<N, R, -1, MINB><<<grid, CT_THREADS, 0, st>>>(B);
}

template <typename R>
int fermion_op_batch(const FopArgs<R>* args, int n, int N, int sign, int sms, cudaStream_t st) {
  if (n < 1 || n > FOP_BATCH_MAX || N < 2 || N > 4 || sms < 1) return -1;
  FopBatch<R> B;
  B.n = n;
  long t = 0;
  for (int i = 0; i < n; i++) {
    if (args[i].trace) return -1;   // the batch forms detLtoS itself
    B.a[i] = args[i];
    B.start[i] = (int)t;
    t += (args[i].g.V + CT_THREADS - 1) / CT_THREADS;
  }
  if (16 * t > 0x7fffffffL) return -1;
  B.tiles = (int)t;
  B.start[n] = (int)t;
  const int resident = (sizeof(R) == 8 ? 4 : 8) * sms;
  const int grid = (int)std::min<long>(16 * t, resident);
  switch (N) {
    case 2: launch_batch<2, R>(B, sign, grid, st); break;
    case 3: launch_batch<3, R>(B, sign, grid, st); break;
    default: launch_batch<4, R>(B, sign, grid, st); break;
  }
  return (int)(16 * t);
}

template int fermion_op_batch<double>(const FopArgs<double>*, int, int, int, int, cudaStream_t);
template int fermion_op_batch<float>(const FopArgs<float>*, int, int, int, int, cudaStream_t);

template <typename R>
int fermion_op_compact(const FopArgs<R>& a, int N, int sign, int variant, cudaStream_t st) {
  switch (variant) {
    case FOP_COMPACT:
    case FOP_COMPACT_PF: {
      const bool pf = variant == FOP_COMPACT_PF;
      switch (N) {
        case 2: return pf ? launch_compact<2, R, true>(a, sign, st) : launch_compact<2, R, false>(a, sign, st);
        case 3: return pf ? launch_compact<3, R, true>(a, sign, st) : launch_compact<3, R, false>(a, sign, st);
        default: return pf ? launch_compact<4, R, true>(a, sign, st) : launch_compact<4, R, false>(a, sign, st);
      }
    }
    case FOP_SITE_MAJOR_PP:
      switch (N) {
        case 2: return launch_pp<2, R, true, true>(a, sign, st);
        case 3: return launch_pp<3, R, true, true>(a, sign, st);
        default: return launch_pp<4, R, true, true>(a, sign, st);
      }
    case FOP_COMP_MAJOR_PP:
      switch (N) {
        case 2: return launch_pp<2, R, false, true>(a, sign, st);
        case 3: return launch_pp<3, R, false, true>(a, sign, st);
        default: return launch_pp<4, R, false, true>(a, sign, st);
      }
    case FOP_SITE_MAJOR:
      switch (N) {
        case 2: return launch_pp<2, R, true, false>(a, sign, st);
        case 3: return launch_pp<3, R, true, false>(a, sign, st);
        default: return launch_pp<4, R, true, false>(a, sign, st);
      }
    case FOP_SITE_MAJOR_OCC:
      switch (N) {
        case 2: return launch_pp<2, R, true, false, 4>(a, sign, st);
        case 3: return launch_pp<3, R, true, false, 4>(a, sign, st);
        default: return launch_pp<4, R, true, false, 4>(a, sign, st);
      }
    case FOP_SITE_MAJOR_SHN:
      switch (N) {
        case 2: return launch_pp<2, R, true, false, 4, true>(a, sign, st);
        case 3: return launch_pp<3, R, true, false, 4, true>(a, sign, st);
        default: return launch_pp<4, R, true, false, 4, true>(a, sign, st);
      }
    case FOP_COMP_MAJOR_SHN:
      switch (N) {
        case 2: return launch_pp<2, R, false, false, 8, true>(a, sign, st);
        case 3: return launch_pp<3, R, false, false, 8, true>(a, sign, st);
        default: return launch_pp<4, R, false, false, 8, true>(a, sign, st);
      }
    case FOP_SITE_MAJOR_FRONT: {
      constexpr int MB = sizeof(R) == 8 ? 4 : 8;
      switch (N) {
        case 2: return launch_pp<2, R, true, false, MB, false, true>(a, sign, st);
        case 3: return launch_pp<3, R, true, false, MB, false, true>(a, sign, st);
        default: return launch_pp<4, R, true, false, MB, false, true>(a, sign, st);
      }
    }
    case FOP_SITE_MAJOR_TR: {
      constexpr int MB = sizeof(R) == 8 ? 4 : 8;
      switch (N) {
        case 2: return launch_pp<2, R, true, false, MB, false, true, true>(a, sign, st);
        case 3: return launch_pp<3, R, true, false, MB, false, true, true>(a, sign, st);
        default: return launch_pp<4, R, true, false, MB, false, true, true>(a, sign, st);
      }
    }
    case FOP_GROUPED:
      switch (N) {
        case 2: return launch_grp<2, R>(a, sign, st);
        case 3: return launch_grp<3, R>(a, sign, st);
        default: return launch_grp<4, R>(a, sign, st);
      }
    default:
      switch (N) {
        case 2: return launch_pp<2, R, false, false, 8>(a, sign, st);
        case 3: return launch_pp<3, R, false, false, 8>(a, sign, st);
        default: return launch_pp<4, R, false, false, 8>(a, sign, st);
      }
  }
}

template int fermion_op_compact<double>(const FopArgs<double>&, int, int, int, cudaStream_t);
template int fermion_op_compact<float>(const FopArgs<float>&, int, int, int, cudaStream_t);

}  // namespace susy
