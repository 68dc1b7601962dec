// Table-driven variant of the fermion operator (same terms as
// fermion_op.cu, 4d_Q16/susy/utilities.c:141-865).
//
// Every one of the 220 NCOL x NCOL products per site is one row of a term
// table in constant memory (coefficient, temporal-BC displacement, and the
// component and neighbour displacement of each factor), grouped by operand
// pattern so that which fields enter and which are adjointed is known at
// compile time.  Neighbour indices come from a per-lattice table
// (tab[d * S + s], one coalesced int per factor) instead of per-term wrap
// arithmetic.  A thread loops over the 10-16 terms of its output matrix,
// optionally with the next term's operands prefetched.  The loop bodies are
// a few hundred instructions, so the instruction working set stays in the
// SM's instruction cache (the fully unrolled kernels stall on instruction
// fetch) and only one or two products' operands are live.  The determinant
// terms (detStoL, detLtoS, G != 0) follow the loops.
#include <mutex>
#include <vector>
#include "common.cuh"
#include "fop.cuh"
#include "kernels.h"

namespace susy {

// Operand patterns: every product is one of
//   P_UF: U * F     P_FU: F * U     P_FUD: F * U^dag     P_UDF: U^dag * F
// (F = the source Twist_Fermion, itself adjointed when sign = -1), so the
// loops run per pattern with compile-time operand fields and adjoints.
enum { P_UF = 0, P_FU = 1, P_FUD = 2, P_UDF = 3, NPAT = 4 };

struct FTerm {
  int8_t kl, dl, kr, dr;   // components and displacement indices of the factors
  int8_t bcdt, pad0, pad1, pad2;
  float coef;
};

constexpr int MAX_TERMS = 224;
constexpr int MAX_DISP = 64;
__constant__ FTerm c_terms[MAX_TERMS];
__constant__ short c_pat_start[NTF][NPAT + 1];
__constant__ char4 c_disp[MAX_DISP];
static int h_ndisp = 0;

// ---------------------------------------------------------------------------
// Host: build the term table once per device
struct TermBuilder {
  std::vector<FTerm> terms[NTF][NPAT];
  std::vector<char4> disp;

  int d(int dx, int dy, int dz, int dt) {
    for (size_t i = 0; i < disp.size(); i++)
      if (disp[i].x == dx && disp[i].y == dy && disp[i].z == dz && disp[i].w == dt) return (int)i;
    disp.push_back(make_char4(dx, dy, dz, dt));
    return (int)disp.size() - 1;
  }
  // displacement of a signed sum of link offsets
  int dl(std::initializer_list<int> plus, std::initializer_list<int> minus = {}) {
    int x = 0, y = 0, z = 0, t = 0;
    for (int a : plus) { x += ex(a); y += ey(a); z += ez(a); t += et(a); }
    for (int a : minus) { x -= ex(a); y -= ey(a); z -= ez(a); t -= et(a); }
    return d(x, y, z, t);
  }
  static int tdt(std::initializer_list<int> plus, std::initializer_list<int> minus = {}) {
    int t = 0;
    for (int a : plus) t += et(a);
    for (int a : minus) t -= et(a);
    return t;
  }
  void add(int comp, int pat, double coef, int bcdt, int kl, int dlv, int kr, int drv) {
    FTerm T;
    T.kl = kl; T.dl = dlv; T.kr = kr; T.dr = drv;
    T.bcdt = bcdt; T.pad0 = T.pad1 = T.pad2 = 0;
    T.coef = (float)coef;
    terms[comp][pat].push_back(T);
  }

  void build() {
    // component 0: eta'  (DbminusLtoS, utilities.c:634-682)
    for (int e = 0; e < 5; e++) {
      add(0, P_FUD, 0.5, 0, 1 + e, dl({}), e, dl({}));
      add(0, P_UDF, -0.5, tdt({}, {e}), e, dl({}, {e}), 1 + e, dl({}, {e}));
    }
    // components 1..5: psi'_B  (Dminus 228-321, DbplusStoL 517-545)
    for (int B = 0; B < 5; B++) {
      for (int e = 0; e < 5; e++) {
        if (e == B) continue;
        const double sg = e < B ? 1.0 : -1.0;
        add(1 + B, P_UF, sg, 0, e, dl({B}), 6 + pidx(e, B), dl({}));
        add(1 + B, P_FU, -sg, tdt({}, {e}), 6 + pidx(e, B), dl({}, {e}), e, dl({}, {e}));
      }
      add(1 + B, P_FUD, 0.5, tdt({B}), 0, dl({B}), B, dl({}));
      add(1 + B, P_UDF, -0.5, 0, B, dl({}), 0, dl({}));
    }
    // components 6..15: chi'_AB  (Dplus 137-221, DbplusPtoP 327-414,
    // DbminusPtoP 420-510)
    for (int A = 0; A < 5; A++)
      for (int B = A + 1; B < 5; B++) {
        const int q = 6 + pidx(A, B);
        add(q, P_UF, 1.0, tdt({A}), A, dl({}), 1 + B, dl({A}));
        add(q, P_FU, -1.0, 0, 1 + B, dl({}), A, dl({B}));
        add(q, P_UF, -1.0, tdt({B}), B, dl({}), 1 + A, dl({B}));
        add(q, P_FU, 1.0, 0, 1 + A, dl({}), B, dl({A}));
        int K[3], k = 0;
        for (int v = 0; v < 5; v++)
          if (v != A && v != B) K[k++] = v;
        for (int ci = 0; ci < 3; ci++) {
          const int C = K[ci];
          const int P = ci == 0 ? K[1] : K[0];
          const int Q = ci == 2 ? K[1] : K[2];
          const int pq = 6 + pidx(P, Q);
          const double t1 = 0.5 * eps5(A, B, C, P, Q), t2 = 0.5 * eps5(P, Q, C, A, B);
          add(q, P_FUD, t1, tdt({A, B, C}), pq, dl({A, B, C}), C, dl({A, B}));
          add(q, P_UDF, -t1, tdt({A, B}), C, dl({}, {C}), pq, dl({A, B}));
          add(q, P_FUD, t2, tdt({}, {P, Q}), pq, dl({}, {P, Q}), C, dl({}, {P, Q, C}));
          add(q, P_UDF, -t2, tdt({}, {P, Q, C}), C, dl({}, {C}), pq, dl({}, {P, Q, C}));
        }
      }
  }
};

static std::mutex g_terms_mu;
static bool g_terms_ready[64];

int upload_fop_terms(int device, cudaStream_t st) {
  (void)st;
  std::lock_guard<std::mutex> lk(g_terms_mu);
  if (device >= 0 && device < 64 && g_terms_ready[device]) return 0;
  TermBuilder tb;
  tb.build();
  std::vector<FTerm> flat;
  short start[NTF][NPAT + 1];
  for (int c = 0; c < NTF; c++)
    for (int p = 0; p < NPAT; p++) {
      start[c][p] = (short)flat.size();
      flat.insert(flat.end(), tb.terms[c][p].begin(), tb.terms[c][p].end());
      start[c][p + 1] = (short)flat.size();
    }
  if ((int)flat.size() > MAX_TERMS || (int)tb.disp.size() > MAX_DISP) return -1;
  cudaMemcpyToSymbol(c_terms, flat.data(), flat.size() * sizeof(FTerm));
  cudaMemcpyToSymbol(c_pat_start, start, sizeof(start));
  cudaMemcpyToSymbol(c_disp, tb.disp.data(), tb.disp.size() * sizeof(char4));
  h_ndisp = (int)tb.disp.size();
  if (cudaGetLastError() != cudaSuccess) return -2;
  if (device >= 0 && device < 64) g_terms_ready[device] = true;
  return 0;
}

int fop_ndisp() { return h_ndisp; }

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
  count_launch(), k_nbr_table<<<(g.V + 127) / 128, 128, 0, st>>>(g, h_ndisp, tab);
}

// ---------------------------------------------------------------------------
// Device
// Temporal BC factors of a thread's site for net displacements -3..3:
// bit (dt + 3) set when t + dt leaves [0, nt - 1]
SUSY_D unsigned bc_mask(const Geo& g, const Site& c) {
  unsigned m = 0;
#pragma unroll
  for (int dt = -3; dt <= 3; dt++) {
    const int t = c.t + dt;
    if (t < 0 || t > g.nt - 1) m |= 1u << (dt + 3);
  }
  return m;
}

template <typename R>
SUSY_D R bc_of(unsigned mask, int dt, R pbc) {
  return ((mask >> (dt + 3)) & 1u) ? pbc : (R)1;
}

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
      mac<0>(acc, (R)T.coef * bc_of<R>(bcm, T.bcdt, pbc), L, Rm);
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
      mac<0>(acc, (R)T.coef * bc_of<R>(bcm, T.bcdt, pbc), L, Rm);
    }
  }
}

// Tr(A op(B)) for A = component ka of fa at site sa and B = component kb of
// fb at site sb (op(B) = B^dag when ADJB), one element pair at a time: the
// determinant terms run while the accumulator is live, and holding whole
// matrices here made the register-capped kernels spill
template <int N, typename R, bool ADJB>
SUSY_D Cx<R> trace_ld(const typename CT<R>::T* fa, int ka, int sa, const typename CT<R>::T* fb,
                      int kb, int sb, int S) {
  const typename CT<R>::T* pa = fa + (size_t)(ka * N * N) * S + sa;
  const typename CT<R>::T* pb = fb + (size_t)(kb * N * N) * S + sb;
  Cx<R> t(0, 0);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int k = 0; k < N; k++) {
      const Cx<R> x = ldc<R>(pa + (size_t)(i * N + k) * S);
      const Cx<R> y = ADJB ? conj(ldc<R>(pb + (size_t)(i * N + k) * S))
                           : ldc<R>(pb + (size_t)(k * N + i) * S);
      t = t + x * y;
    }
  return t;
}

// detStoL for output link B (utilities.c:551-628)
template <int N, typename R, int SIGN>
SUSY_D void det_stol_rt(Mat<N, R>& acc, const FopArgs<R>& a, const Site& c, int B) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  Cx<R> tsum(0, 0);
  const Cx<R> tr0 = ldtr<N, R, ADJ>(a.src, 0, s, S);
#pragma unroll 1
  for (int e = 0; e < NUMLINK; e++) {
    if (e == B) continue;
    const int mE = nbr(g, c, -ex(e), -ey(e), -ez(e), -et(e));
    tsum = tsum + tr0 * ldc<R>(a.pd + (size_t)(e * 5 + B) * S + s);
    const Cx<R> trm = ldtr<N, R, ADJ>(a.src, 0, mE, S);
    tsum = tsum + bcf<R>(g, c, -et(e)) * (trm * ldc<R>(a.pd + (size_t)(B * 5 + e) * S + mE));
  }
  const Cx<R> f = ((R)(-0.5) * a.G) * tsum;
  const typename CT<R>::T* pu = a.Uinv + (size_t)(B * N * N) * S + s;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) acc.e[i][j] = acc.e[i][j] + f * ldc<R>(pu + (size_t)(i * N + j) * S);
}

// detLtoS for the site output (utilities.c:688-756)
template <int N, typename R, int SIGN>
SUSY_D void det_ltos_rt(Mat<N, R>& acc, const FopArgs<R>& a, const Site& c) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  Cx<R> T0[NUMLINK];
#pragma unroll
  for (int e = 0; e < NUMLINK; e++) T0[e] = trace_ld<N, R, ADJ>(a.Uinv, e, s, a.src, 1 + e, s, S);
  Cx<R> tsum(0, 0);
#pragma unroll 1
  for (int b = 0; b < NUMLINK; b++) {
    const int pb = nbr(g, c, ex(b), ey(b), ez(b), et(b));
    const R bcb = bcf<R>(g, c, et(b));
    Cx<R> T0b = T0[0];
#pragma unroll
    for (int e = 1; e < NUMLINK; e++)
      if (e == b) T0b = T0[e];
#pragma unroll 1
    for (int e = 0; e < NUMLINK; e++) {
      if (e == b) continue;
      const Cx<R> Tp = trace_ld<N, R, ADJ>(a.Uinv, e, pb, a.src, 1 + e, pb, S);
      tsum = tsum + ldc<R>(a.pd + (size_t)(e * 5 + b) * S + s) * (T0b + bcb * Tp);
    }
  }
  const Cx<R> d = ((R)0.5 * a.G) * tsum;
#pragma unroll
  for (int i = 0; i < N; i++) acc.e[i][i] = acc.e[i][i] + d;
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

// Shared epilogue: determinant terms, adjoint for D^dag, axpy and dot
template <int N, typename R, int SIGN>
SUSY_D double fop_finish(Mat<N, R>& acc, const FopArgs<R>& a, const Site& c, int comp) {
  if (a.doG) {
    if (comp == 0)
      det_ltos_rt<N, R, SIGN>(acc, a, c);
    else if (comp <= NUMLINK)
      det_stol_rt<N, R, SIGN>(acc, a, c, comp - 1);
  }
  if (SIGN < 0) {
    Mat<N, R> t = acc;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) acc.e[i][j] = Cx<R>(-t.e[j][i].re, t.e[j][i].im);
  }
  double part = 0.0;
  if (a.add) {
    Mat<N, R> x = ldm<N, R>(a.add, comp, c.s, a.g.S);
    axpy(acc, Cx<R>(a.addc, 0), x);
    if (a.dot) part = rdot(x, acc);
  }
  stm<N, R>(a.dst, comp, c.s, a.g.S, acc);
  return part;
}

// PP = false: one operand buffer, no prefetch (fewest registers)
template <int N, typename R, int SIGN, int PAT, bool PP, typename ACC>
SUSY_D void run_pattern_pp(ACC& acc, const FopArgs<R>& a, int s, unsigned bcm, int t0, int t1) {
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
      const Mat<N, R> L = ldm<N, R, AL>(fl, T.kl, a.nbrtab[(size_t)T.dl * S + s], S);
      const Mat<N, R> Rm = ldm<N, R, AR>(fr, T.kr, a.nbrtab[(size_t)T.dr * S + s], S);
      acc.add((R)T.coef * bc_of<R>(bcm, T.bcdt, pbc), L, Rm);
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
    acc.add((R)TA.coef * bc_of<R>(bcm, TA.bcdt, pbc), LA, RA);
    if (!hb) break;
    const bool ha = t + 2 < t1;
    if (ha) {
      TA = c_terms[t + 2];
      LA = ldm<N, R, AL>(fl, TA.kl, a.nbrtab[(size_t)TA.dl * S + s], S);
      RA = ldm<N, R, AR>(fr, TA.kr, a.nbrtab[(size_t)TA.dr * S + s], S);
    }
    acc.add((R)TB.coef * bc_of<R>(bcm, TB.bcdt, pbc), LB, RB);
    if (!ha) break;
  }
}

// Block order: site-major (SM = true) or component-major; PP: two operand
// buffers (prefetch) or one.
template <int N, typename R, int SIGN, bool SM, bool PP, int MINB>
__global__ void __launch_bounds__(CT_THREADS, MINB)
fermion_op_pp_kernel(FopArgs<R> a) {
  if (a.skip && *a.skip) return;
  const int comp = SM ? blockIdx.x % NTF : blockIdx.x / a.nsb;
  const int s = (SM ? blockIdx.x / NTF : blockIdx.x % a.nsb) * CT_THREADS + threadIdx.x;
  double part = 0.0;
  if (s < a.g.V) {
    const Site c = site_of(a.g, s);
    const unsigned bcm = bc_mask(a.g, c);
    AccMat<N, R> acc;
    acc.zero();
    run_pattern_pp<N, R, SIGN, P_UF, PP>(acc, a, s, bcm, c_pat_start[comp][0], c_pat_start[comp][1]);
    run_pattern_pp<N, R, SIGN, P_FU, PP>(acc, a, s, bcm, c_pat_start[comp][1], c_pat_start[comp][2]);
    run_pattern_pp<N, R, SIGN, P_FUD, PP>(acc, a, s, bcm, c_pat_start[comp][2], c_pat_start[comp][3]);
    run_pattern_pp<N, R, SIGN, P_UDF, PP>(acc, a, s, bcm, c_pat_start[comp][3], c_pat_start[comp][4]);
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

template <int N, typename R, bool SM, bool PP, int MINB = 1>
static int launch_pp(FopArgs<R> a, int sign, cudaStream_t st) {
  a.nsb = (a.g.V + CT_THREADS - 1) / CT_THREADS;
  const int nblk = a.nsb * NTF;
  if (sign > 0)
    count_launch(), fermion_op_pp_kernel<N, R, 1, SM, PP, MINB><<<nblk, CT_THREADS, 0, st>>>(a);
  else
    count_launch(), fermion_op_pp_kernel<N, R, -1, SM, PP, MINB><<<nblk, CT_THREADS, 0, st>>>(a);
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
