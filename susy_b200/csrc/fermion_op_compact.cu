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

// Block order: site-major (SM = true) or component-major; PP: two operand
// buffers (prefetch) or one.
// SHN: the block first copies its output component's neighbour indices
// (at most MAX_SLOTS displacements x CT_THREADS sites) into shared memory,
// so a product's operand loads no longer wait on a global index load.
template <int N, typename R, int SIGN, bool SM, bool PP, int MINB, bool SHN = false>
__global__ void __launch_bounds__(CT_THREADS, MINB)
fermion_op_pp_kernel(FopArgs<R> a) {
  if (a.skip && *a.skip) return;
  const int comp = SM ? blockIdx.x % NTF : blockIdx.x / a.nsb;
  const int s = (SM ? blockIdx.x / NTF : blockIdx.x % a.nsb) * CT_THREADS + threadIdx.x;
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
    part = fop_finish<N, R, SIGN>(out, a, c, comp);
  }
  if (a.dot) {
    part = block_sum<CT_THREADS>(part);
    if (threadIdx.x == 0) a.dot[blockIdx.x] = part;
  }
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

template <int N, typename R, bool SM, bool PP, int MINB = 1, bool SHN = false>
static int launch_pp(FopArgs<R> a, int sign, cudaStream_t st) {
  a.nsb = (a.g.V + CT_THREADS - 1) / CT_THREADS;
  const int nblk = a.nsb * NTF;
  if (sign > 0)
    count_launch(), fermion_op_pp_kernel<N, R, 1, SM, PP, MINB, SHN><<<nblk, CT_THREADS, 0, st>>>(a);
  else
    count_launch(), fermion_op_pp_kernel<N, R, -1, SM, PP, MINB, SHN><<<nblk, CT_THREADS, 0, st>>>(a);
  return nblk;
}

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
