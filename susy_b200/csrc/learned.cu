// Learned preconditioner: a gauge-covariant network of parallel-transported
// nearest-neighbour convolutions (no reference counterpart; the CPU
// definition and its gradient checks are oracle/learned_np.py).
//
//   embed      Twist_Fermion -> 16 site-type channels:
//              S_0 = eta, S_{1+a} = psi_a U_a^-1,
//              S_{6+p(a,b)} = chi_ab U_b(x+a)^-1 U_a(x)^-1
//   3 layers   16 -> 32 -> 32 -> 16 channels,
//              out_c(x) = sum_{k,c'} W[k][c][c'] T_k(in_c')(x) over the 11
//              transports T_0 X = X, T_{1+mu} X = U_mu X(x+mu) U_mu^-1,
//              T_{6+mu} X = U_mu(x-mu)^-1 X(x-mu) U_mu(x-mu)
//   unembed    the inverse of embed
//
// Weights are bfloat16 pairs (re, im) on the device; every product and sum
// is FP32 (the channels, the transports, the accumulators); the network's
// input and output are FP64 Twist_Fermions in the device layout.  Channel
// fields use the device layout with K = channels (float2).
//
// Kernels per layer: k_transport (thread per site and channel, the 10
// matrix triple products), k_mix (thread per matrix element row of the
// [sites x N^2] x [11 Cin] transport matrix, all Cout accumulators in
// registers; the weights are read with warp-uniform addresses and so are
// broadcast from L1).  Backward: k_mix_adj (same shape, conjugate weights),
// k_transport_adj (the adjoint transports), k_wgrad (weight gradient: a
// block per tap row k and row chunk, partial sums over rows, summed in FP64
// on the host).
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>
#include "hmc.h"
#include "lattice.h"

namespace susy {

constexpr int NT_TAP = 11;
constexpr int LT = 128;

// ---------------------------------------------------------------------------
// Matrix helpers on FP32 complex matrices
template <int N>
SUSY_D Mat<N, float> ldmf(const float2* f, int k, int s, int S) { return ldm<N, float>(f, k, s, S); }

template <int N>
SUSY_D Mat<N, float> mulf(const Mat<N, float>& A, const Mat<N, float>& B) {
  return mul(A, B);
}

template <int N>
SUSY_D Mat<N, float> adjf(const Mat<N, float>& A) { return adjm(A); }

template <int N>
SUSY_D Mat<N, float> to32(const Mat<N, double>& A) {
  Mat<N, float> m;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) m.e[i][j] = Cx<float>((float)A.e[i][j].re, (float)A.e[i][j].im);
  return m;
}

template <int N>
SUSY_D Mat<N, double> to64(const Mat<N, float>& A) {
  Mat<N, double> m;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) m.e[i][j] = Cx<double>(A.e[i][j].re, A.e[i][j].im);
  return m;
}

// ---------------------------------------------------------------------------
// embed / unembed / adjoint of unembed: one thread per site
template <int N>
__global__ void __launch_bounds__(LT) k_embed(Geo g, const float2* U, const float2* Ui,
                                              const double2* tf, float2* X) {
  const int s = blockIdx.x * LT + threadIdx.x;
  if (s >= g.V) return;
  const int S = g.S;
  const Site c = site_of(g, s);
  stm<N, float>(X, 0, s, S, to32<N>(ldm<N, double>(tf, 0, s, S)));
#pragma unroll 1
  for (int a = 0; a < NUMLINK; a++)
    stm<N, float>(X, 1 + a, s, S, mulf<N>(to32<N>(ldm<N, double>(tf, 1 + a, s, S)), ldmf<N>(Ui, a, s, S)));
#pragma unroll 1
  for (int a = 0; a < NUMLINK; a++)
#pragma unroll 1
    for (int b = a + 1; b < NUMLINK; b++) {
      const int p = pidx(a, b);
      const int xa = nbr(g, c, ex(a), ey(a), ez(a), et(a));
      const Mat<N, float> w = mulf<N>(ldmf<N>(Ui, b, xa, S), ldmf<N>(Ui, a, s, S));
      stm<N, float>(X, 6 + p, s, S, mulf<N>(to32<N>(ldm<N, double>(tf, 6 + p, s, S)), w));
    }
}

template <int N>
__global__ void __launch_bounds__(LT) k_unembed(Geo g, const float2* U, const float2* X,
                                                double2* tf) {
  const int s = blockIdx.x * LT + threadIdx.x;
  if (s >= g.V) return;
  const int S = g.S;
  const Site c = site_of(g, s);
  stm<N, double>(tf, 0, s, S, to64<N>(ldmf<N>(X, 0, s, S)));
#pragma unroll 1
  for (int a = 0; a < NUMLINK; a++)
    stm<N, double>(tf, 1 + a, s, S, to64<N>(mulf<N>(ldmf<N>(X, 1 + a, s, S), ldmf<N>(U, a, s, S))));
#pragma unroll 1
  for (int a = 0; a < NUMLINK; a++)
#pragma unroll 1
    for (int b = a + 1; b < NUMLINK; b++) {
      const int p = pidx(a, b);
      const int xa = nbr(g, c, ex(a), ey(a), ez(a), et(a));
      const Mat<N, float> w = mulf<N>(ldmf<N>(U, a, s, S), ldmf<N>(U, b, xa, S));
      stm<N, double>(tf, 6 + p, s, S, to64<N>(mulf<N>(ldmf<N>(X, 6 + p, s, S), w)));
    }
}

// gX = unembed^dag(G) for an FP64 gradient G scaled by sc
template <int N>
__global__ void __launch_bounds__(LT) k_unembed_adj(Geo g, const float2* U, const double2* G,
                                                    double sc, float2* X) {
  const int s = blockIdx.x * LT + threadIdx.x;
  if (s >= g.V) return;
  const int S = g.S;
  const Site c = site_of(g, s);
  auto ldg = [&](int k) {
    Mat<N, float> m = to32<N>(ldm<N, double>(G, k, s, S));
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) m.e[i][j] = Cx<float>((float)sc * m.e[i][j].re, (float)sc * m.e[i][j].im);
    return m;
  };
  stm<N, float>(X, 0, s, S, ldg(0));
#pragma unroll 1
  for (int a = 0; a < NUMLINK; a++)
    stm<N, float>(X, 1 + a, s, S, mulf<N>(ldg(1 + a), adjf<N>(ldmf<N>(U, a, s, S))));
#pragma unroll 1
  for (int a = 0; a < NUMLINK; a++)
#pragma unroll 1
    for (int b = a + 1; b < NUMLINK; b++) {
      const int p = pidx(a, b);
      const int xa = nbr(g, c, ex(a), ey(a), ez(a), et(a));
      const Mat<N, float> w = mulf<N>(ldmf<N>(U, a, s, S), ldmf<N>(U, b, xa, S));
      stm<N, float>(X, 6 + p, s, S, mulf<N>(ldg(6 + p), adjf<N>(w)));
    }
}

// ---------------------------------------------------------------------------
// transports: T[k][c] for k = 0..10 (thread per site and channel)
template <int N>
__global__ void __launch_bounds__(LT) k_transport(Geo g, const float2* U, const float2* Ui,
                                                  const float2* X, int C, float2* T) {
  const int s = blockIdx.x * LT + threadIdx.x;
  const int ch = blockIdx.y;
  if (s >= g.V) return;
  const int S = g.S;
  const Site c = site_of(g, s);
  const size_t cs = (size_t)C;   // channels per tap
  stm<N, float>(T, ch, s, S, ldmf<N>(X, ch, s, S));
#pragma unroll 1
  for (int mu = 0; mu < NUMLINK; mu++) {
    const int xp = nbr(g, c, ex(mu), ey(mu), ez(mu), et(mu));
    const int xm = nbr(g, c, -ex(mu), -ey(mu), -ez(mu), -et(mu));
    const Mat<N, float> f = mulf<N>(mulf<N>(ldmf<N>(U, mu, s, S), ldmf<N>(X, ch, xp, S)),
                                    ldmf<N>(Ui, mu, s, S));
    stm<N, float>(T + (1 + mu) * cs * N * N * S, ch, s, S, f);
    const Mat<N, float> b = mulf<N>(mulf<N>(ldmf<N>(Ui, mu, xm, S), ldmf<N>(X, ch, xm, S)),
                                    ldmf<N>(U, mu, xm, S));
    stm<N, float>(T + (6 + mu) * cs * N * N * S, ch, s, S, b);
  }
}

// gX[c] = sum_k T_k^dag(gT[k][c])
template <int N>
__global__ void __launch_bounds__(LT) k_transport_adj(Geo g, const float2* U, const float2* Ui,
                                                      const float2* gT, int C, float2* gX) {
  const int s = blockIdx.x * LT + threadIdx.x;
  const int ch = blockIdx.y;
  if (s >= g.V) return;
  const int S = g.S;
  const Site c = site_of(g, s);
  const size_t tap = (size_t)C * N * N * S;
  Mat<N, float> acc = ldmf<N>(gT, ch, s, S);
#pragma unroll 1
  for (int mu = 0; mu < NUMLINK; mu++) {
    const int xp = nbr(g, c, ex(mu), ey(mu), ez(mu), et(mu));
    const int xm = nbr(g, c, -ex(mu), -ey(mu), -ez(mu), -et(mu));
    // forward tap: U(y-mu)^dag G(y-mu) U(y-mu)^-dag
    Mat<N, float> t = mulf<N>(mulf<N>(adjf<N>(ldmf<N>(U, mu, xm, S)),
                                      ldmf<N>(gT + (1 + mu) * tap, ch, xm, S)),
                              adjf<N>(ldmf<N>(Ui, mu, xm, S)));
    // backward tap: U(y)^-dag G(y+mu) U(y)^dag
    Mat<N, float> u = mulf<N>(mulf<N>(adjf<N>(ldmf<N>(Ui, mu, s, S)),
                                      ldmf<N>(gT + (6 + mu) * tap, ch, xp, S)),
                              adjf<N>(ldmf<N>(U, mu, s, S)));
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) acc.e[i][j] = acc.e[i][j] + t.e[i][j] + u.e[i][j];
  }
  stm<N, float>(gX, ch, s, S, acc);
}

// ---------------------------------------------------------------------------
// Channel mixing.  Rows r = (element, site) of a channel field (M = N^2 S
// rows per channel); T is [K][M] with K = 11 Cin, out [Cout][M].
SUSY_D float2 wload(const uint32_t* W, int idx) {
  const uint32_t v = W[idx];
  __nv_bfloat16_raw lo, hi;
  lo.x = (unsigned short)(v & 0xffffu);
  hi.x = (unsigned short)(v >> 16);
  return make_float2(__bfloat162float(__nv_bfloat16(lo)), __bfloat162float(__nv_bfloat16(hi)));
}

template <int COUT>
__global__ void __launch_bounds__(LT) k_mix(long M, int K, const float2* T, const uint32_t* W,
                                            float2* out) {
  const long r = (long)blockIdx.x * LT + threadIdx.x;
  if (r >= M) return;
  float2 acc[COUT];
#pragma unroll
  for (int c = 0; c < COUT; c++) acc[c] = make_float2(0.f, 0.f);
#pragma unroll 1
  for (int k = 0; k < K; k++) {
    const float2 t = T[(size_t)k * M + r];
#pragma unroll
    for (int c = 0; c < COUT; c++) {
      const float2 w = wload(W, k * COUT + c);
      acc[c].x = fmaf(w.x, t.x, fmaf(-w.y, t.y, acc[c].x));
      acc[c].y = fmaf(w.x, t.y, fmaf(w.y, t.x, acc[c].y));
    }
  }
#pragma unroll
  for (int c = 0; c < COUT; c++) out[(size_t)c * M + r] = acc[c];
}

// gT[k][r] = sum_c conj(W[k][c]) g[c][r]
template <int COUT>
__global__ void __launch_bounds__(LT) k_mix_adj(long M, int K, const float2* gOut,
                                                const uint32_t* W, float2* gT) {
  const long r = (long)blockIdx.x * LT + threadIdx.x;
  if (r >= M) return;
  float2 gv[COUT];
#pragma unroll
  for (int c = 0; c < COUT; c++) gv[c] = gOut[(size_t)c * M + r];
#pragma unroll 1
  for (int k = 0; k < K; k++) {
    float2 a = make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < COUT; c++) {
      const float2 w = wload(W, k * COUT + c);
      a.x = fmaf(w.x, gv[c].x, fmaf(w.y, gv[c].y, a.x));
      a.y = fmaf(w.x, gv[c].y, fmaf(-w.y, gv[c].x, a.y));
    }
    gT[(size_t)k * M + r] = a;
  }
}

// Channel mixing on the tensor cores (inference): the complex product
// out[c][r] = sum_k W[k][c] T[k][r] as the real GEMM
//   [M rows x 2K] x [2K x 2 Cout],  A[r][2k + p] = (Re, Im)_p T[k][r],
//   B[2k + p][2c + q] = {{Re W, Im W}, {-Im W, Re W}}[p][q],
// with mma.m16n8k16 (BF16 inputs, FP32 accumulation).  With (Re, Im) of a
// complex element adjacent along K, every A-fragment register of a thread
// is one transport element T[k][r] rounded to a bf16 pair, and every pair
// of accumulator registers is (Re, Im) of one output channel.  The B
// fragments are packed by the host (net_set_weights) in the order a warp
// reads them: Wp[(step * NT + tile) * 32 + lane] = {b0, b1}.  One warp per
// 16 rows, all output channels; rows past M read zeros and store nothing.
SUSY_D uint32_t bf16x2(float2 v) {
  const __nv_bfloat162 b = __floats2bfloat162_rn(v.x, v.y);
  uint32_t u;
  memcpy(&u, &b, 4);
  return u;
}

template <int COUT>
__global__ void __launch_bounds__(128) k_mix_mma(long M, int K, const float2* T, const uint2* Wp,
                                                 float2* out) {
  constexpr int NT = COUT / 4;        // n8 tiles of the 2 COUT real columns
  const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
  const long r0 = ((long)blockIdx.x * 4 + (threadIdx.x >> 5)) * 16;
  if (r0 >= M) return;
  const long ra = r0 + gid, rb = r0 + gid + 8;
  const bool oka = ra < M, okb = rb < M;
  float acc[NT][4];
#pragma unroll
  for (int t = 0; t < NT; t++) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.f;
  const float2 z = make_float2(0.f, 0.f);
  const int steps = K / 8;            // 16 real K values = 8 complex ones per step
#pragma unroll 1
  for (int st = 0; st < steps; st++) {
    const float2* t0 = T + (size_t)(8 * st + tig) * M;
    const float2* t4 = T + (size_t)(8 * st + tig + 4) * M;
    const uint32_t a0 = bf16x2(oka ? t0[ra] : z), a1 = bf16x2(okb ? t0[rb] : z);
    const uint32_t a2 = bf16x2(oka ? t4[ra] : z), a3 = bf16x2(okb ? t4[rb] : z);
    const uint2* wp = Wp + (size_t)st * NT * 32 + lane;
#pragma unroll
    for (int t = 0; t < NT; t++) {
      const uint2 b = __ldg(wp + t * 32);
      asm volatile(
          "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
          "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
          : "+f"(acc[t][0]), "+f"(acc[t][1]), "+f"(acc[t][2]), "+f"(acc[t][3])
          : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b.x), "r"(b.y));
    }
  }
#pragma unroll
  for (int t = 0; t < NT; t++) {
    const int c = 4 * t + tig;
    if (oka) out[(size_t)c * M + ra] = make_float2(acc[t][0], acc[t][1]);
    if (okb) out[(size_t)c * M + rb] = make_float2(acc[t][2], acc[t][3]);
  }
}

// partial[rb][k][c] = sum over rows of chunk rb of conj(T[k][r]) g[c][r]
template <int COUT>
__global__ void __launch_bounds__(LT) k_wgrad(long M, int K, const float2* T, const float2* gOut,
                                              long rows_per_block, double2* partial) {
  const int k = blockIdx.x;
  const int rb = blockIdx.y;
  const long r0 = (long)rb * rows_per_block;
  const long r1 = r0 + rows_per_block < M ? r0 + rows_per_block : M;
  float2 acc[COUT];
#pragma unroll
  for (int c = 0; c < COUT; c++) acc[c] = make_float2(0.f, 0.f);
  for (long r = r0 + threadIdx.x; r < r1; r += LT) {
    const float2 t = T[(size_t)k * M + r];
#pragma unroll
    for (int c = 0; c < COUT; c++) {
      const float2 gv = gOut[(size_t)c * M + r];
      acc[c].x = fmaf(t.x, gv.x, fmaf(t.y, gv.y, acc[c].x));
      acc[c].y = fmaf(t.x, gv.y, fmaf(-t.y, gv.x, acc[c].y));
    }
  }
  __shared__ double2 red[LT / 32][COUT];
#pragma unroll
  for (int c = 0; c < COUT; c++) {
    double x = acc[c].x, y = acc[c].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      y += __shfl_xor_sync(0xffffffffu, y, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][c] = make_double2(x, y);
  }
  __syncthreads();
  if (threadIdx.x < COUT) {
    double x = 0.0, y = 0.0;
    for (int w = 0; w < LT / 32; w++) {
      x += red[w][threadIdx.x].x;
      y += red[w][threadIdx.x].y;
    }
    partial[((size_t)rb * K + k) * COUT + threadIdx.x] = make_double2(x, y);
  }
}

// d = z - e (FP64), partials of |d|^2 and |e|^2
__global__ void __launch_bounds__(256) k_diff(long n, const double2* z, const double2* e,
                                              double2* d, double* part) {
  const long i = (long)blockIdx.x * 256 + threadIdx.x;
  double a = 0.0, b = 0.0;
  if (i < n) {
    const double2 zz = z[i], ee = e[i];
    const double2 dd = make_double2(zz.x - ee.x, zz.y - ee.y);
    d[i] = dd;
    a = dd.x * dd.x + dd.y * dd.y;
    b = ee.x * ee.x + ee.y * ee.y;
  }
  a = block_sum<256>(a);
  __syncthreads();
  b = block_sum<256>(b);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

}  // namespace susy

// ---------------------------------------------------------------------------
// Host side
using namespace susy;

static const int kChan[4] = {16, 32, 32, 16};

struct susy_b200_net {
  susy_b200_lattice* h = nullptr;
  uint32_t* W[3] = {};            // bf16 pairs, [11 Cin][Cout] per layer
  uint2* Wp[3] = {};              // the same weights as k_mix_mma's B fragments
  int tc = 1;                     // net_apply mixes on the tensor cores
  float2* X[4] = {};              // channel fields: input of each layer, output
  float2* T[3] = {};              // transports of each layer's input
  float2* gA = nullptr;           // gradient w.r.t. a layer's output / input
  float2* gB = nullptr;
  float2* gT = nullptr;
  double2* tfz = nullptr;         // network output (FP64 Twist_Fermion)
  double2* tfd = nullptr;         // z - e
  double2* wpart = nullptr;       // weight-gradient partials
  double* part = nullptr;
  int rb = 0;                     // row chunks of the weight gradient
  long rows_per_block = 0;
};

static long net_rows(const susy_b200_lattice* h) { return (long)h->N * h->N * h->g.S; }

static int net_kw(int l) { return NT_TAP * kChan[l] * kChan[l + 1]; }
// B-fragment entries of layer l (uint2 each): K / 8 steps x Cout / 4 tiles x 32 lanes
static size_t net_kwp(int l) { return (size_t)(NT_TAP * kChan[l] / 8) * (kChan[l + 1] / 4) * 32; }

extern "C" int susy_b200_net_nweights(void) { return net_kw(0) + net_kw(1) + net_kw(2); }

extern "C" susy_b200_net* susy_b200_net_create(susy_b200_lattice* h) {
  if (!h) return nullptr;
  susy_b200_net* n = new susy_b200_net;
  n->h = h;
  const long M = net_rows(h);
  bool ok = true;
  for (int l = 0; l < 3; l++) {
    n->W[l] = (uint32_t*)dalloc(h, (size_t)net_kw(l) * sizeof(uint32_t));
    n->Wp[l] = (uint2*)dalloc(h, net_kwp(l) * sizeof(uint2));
    ok = ok && n->Wp[l];
    n->T[l] = (float2*)dalloc(h, (size_t)NT_TAP * kChan[l] * M * sizeof(float2));
    ok = ok && n->W[l] && n->T[l];
  }
  for (int l = 0; l < 4; l++) {
    n->X[l] = (float2*)dalloc(h, (size_t)kChan[l] * M * sizeof(float2));
    ok = ok && n->X[l];
  }
  n->gA = (float2*)dalloc(h, (size_t)32 * M * sizeof(float2));
  n->gB = (float2*)dalloc(h, (size_t)32 * M * sizeof(float2));
  n->gT = (float2*)dalloc(h, (size_t)NT_TAP * 32 * M * sizeof(float2));
  n->tfz = (double2*)dalloc(h, field_bytes(h, NTF, 64));
  n->tfd = (double2*)dalloc(h, field_bytes(h, NTF, 64));
  n->rb = (int)std::min<long>(64, (M + 4095) / 4096);
  n->rows_per_block = (M + n->rb - 1) / n->rb;
  n->wpart = (double2*)dalloc(h, (size_t)n->rb * 352 * 32 * sizeof(double2));
  n->part = (double*)dalloc(h, (size_t)2 * (16 * M + 255) / 256 * sizeof(double) + 64);
  ok = ok && n->gA && n->gB && n->gT && n->tfz && n->tfd && n->wpart && n->part;
  if (!ok) {
    susy_b200_net_destroy(n);
    return nullptr;
  }
  return n;
}

// Frees device memory only (cudaFree waits for the device): it must not
// touch the lattice handle, which a caller may already have destroyed
extern "C" void susy_b200_net_destroy(susy_b200_net* n) {
  if (!n) return;
  for (int l = 0; l < 3; l++) {
    if (n->W[l]) cudaFree(n->W[l]);
    if (n->Wp[l]) cudaFree(n->Wp[l]);
    if (n->T[l]) cudaFree(n->T[l]);
  }
  for (int l = 0; l < 4; l++)
    if (n->X[l]) cudaFree(n->X[l]);
  void* ps[] = {n->gA, n->gB, n->gT, n->tfz, n->tfd, n->wpart, n->part};
  for (void* p : ps)
    if (p) cudaFree(p);
  delete n;
}

// Round to bfloat16, nearest even (the host rounding the oracle mirrors)
static uint16_t to_bf16(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  b += 0x7fffu + ((b >> 16) & 1u);
  return (uint16_t)(b >> 16);
}

// w: all layers' weights, complex interleaved, layer by layer, each as
// W[k][c_out][c_in] (the oracle's order); stored transposed per tap row
// ([k c_in][c_out]) for k_mix
extern "C" int susy_b200_net_set_weights(susy_b200_net* n, const double* w) {
  if (!n || !w) return SUSY_B200_EINVAL;
  size_t off = 0;
  for (int l = 0; l < 3; l++) {
    const int ci = kChan[l], co = kChan[l + 1];
    std::vector<uint32_t> hw((size_t)net_kw(l));
    for (int k = 0; k < NT_TAP; k++)
      for (int d = 0; d < co; d++)
        for (int c = 0; c < ci; c++) {
          const size_t src = off + 2 * (((size_t)k * co + d) * ci + c);
          const uint32_t re = to_bf16((float)w[src]), im = to_bf16((float)w[src + 1]);
          hw[((size_t)k * ci + c) * co + d] = re | (im << 16);
        }
    cudaMemcpyAsync(n->W[l], hw.data(), hw.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                    n->h->stream);
    // B fragments of k_mix_mma: lane (gid, tig) of tile t, step st holds
    // B[2k + p][nr], nr = 8 t + gid (output channel nr / 2, Re or Im by
    // nr % 2), k = 8 st + tig (b0) and + 4 (b1), p = 0, 1 in the low and
    // high halves; B = {{Re W, Im W}, {-Im W, Re W}}[p][nr % 2]
    const int steps = NT_TAP * ci / 8, nt = co / 4;
    std::vector<uint2> hp(net_kwp(l));
    auto wpair = [&](int kk, int d, int q) -> uint32_t {
      const int k = kk / ci, c = kk % ci;
      const size_t src = off + 2 * (((size_t)k * co + d) * ci + c);
      const uint16_t wr = to_bf16((float)w[src]), wi = to_bf16((float)w[src + 1]);
      const uint16_t lo = q ? wi : wr;
      const uint16_t hi = q ? wr : (uint16_t)(wi ^ 0x8000u);
      return (uint32_t)lo | ((uint32_t)hi << 16);
    };
    for (int st = 0; st < steps; st++)
      for (int t = 0; t < nt; t++)
        for (int lane = 0; lane < 32; lane++) {
          const int gid = lane >> 2, tig = lane & 3, nr = 8 * t + gid;
          uint2 b;
          b.x = wpair(8 * st + tig, nr >> 1, nr & 1);
          b.y = wpair(8 * st + tig + 4, nr >> 1, nr & 1);
          hp[((size_t)st * nt + t) * 32 + lane] = b;
        }
    cudaMemcpyAsync(n->Wp[l], hp.data(), hp.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                    n->h->stream);
    if (!ck(n->h, cudaStreamSynchronize(n->h->stream))) return SUSY_B200_ECUDA;
    off += 2 * (size_t)net_kw(l);
  }
  return SUSY_B200_OK;
}

// tc: channel mixes on the tensor cores (BF16 transports) or in FP32
template <int N>
static void forward_n(susy_b200_net* n, const void* src, void* dst, bool tc) {
  susy_b200_lattice* h = n->h;
  const Geo& g = h->g;
  const int nb = (g.V + LT - 1) / LT;
  const long M = net_rows(h);
  const int mb = (int)((M + LT - 1) / LT);
  cudaStream_t s = h->stream;
  count_launch(), k_embed<N><<<nb, LT, 0, s>>>(g, (const float2*)h->U32, (const float2*)h->Uinv32,
                                               (const double2*)src, n->X[0]);
  for (int l = 0; l < 3; l++) {
    count_launch(), k_transport<N><<<dim3(nb, kChan[l]), LT, 0, s>>>(
        g, (const float2*)h->U32, (const float2*)h->Uinv32, n->X[l], kChan[l], n->T[l]);
    const int K = NT_TAP * kChan[l];
    const int wb = (int)((M + 63) / 64);   // 4 warps of 16 rows per block
    if (tc && kChan[l + 1] == 32)
      count_launch(), k_mix_mma<32><<<wb, 128, 0, s>>>(M, K, n->T[l], n->Wp[l], n->X[l + 1]);
    else if (tc)
      count_launch(), k_mix_mma<16><<<wb, 128, 0, s>>>(M, K, n->T[l], n->Wp[l], n->X[l + 1]);
    else if (kChan[l + 1] == 32)
      count_launch(), k_mix<32><<<mb, LT, 0, s>>>(M, K, n->T[l], n->W[l], n->X[l + 1]);
    else
      count_launch(), k_mix<16><<<mb, LT, 0, s>>>(M, K, n->T[l], n->W[l], n->X[l + 1]);
  }
  count_launch(), k_unembed<N><<<nb, LT, 0, s>>>(g, (const float2*)h->U32, n->X[3], (double2*)dst);
}

static void net_forward(susy_b200_net* n, const void* src, void* dst, bool tc) {
  switch (n->h->N) {
    case 2: forward_n<2>(n, src, dst, tc); break;
    case 3: forward_n<3>(n, src, dst, tc); break;
    default: forward_n<4>(n, src, dst, tc); break;
  }
}

namespace susy {
// z = N(r) on FP64 device Twist_Fermions (used by the preconditioned solver)
int net_apply(susy_b200_net* n, const void* src, void* dst) {
  net_forward(n, src, dst, n->tc != 0);
  return ck(n->h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}
}  // namespace susy

extern "C" int susy_b200_net_tensor_cores(susy_b200_net* n, int on) {
  if (!n || on > 1) return SUSY_B200_EINVAL;
  const int prev = n->tc;
  if (on >= 0) n->tc = on;
  return prev;
}

extern "C" int susy_b200_net_apply(susy_b200_net* n, const void* src, void* dst) {
  if (!n || !src || !dst) return SUSY_B200_EINVAL;
  return net_apply(n, src, dst);
}

// One layer of the backward pass: weight-gradient partials of layer l into
// wpart; when l > 0 also the gradient w.r.t. the layer's input into gin
template <int N>
static void backward_layer(susy_b200_net* n, int l, const float2* gout, float2* gin) {
  susy_b200_lattice* h = n->h;
  const Geo& g = h->g;
  const int nb = (g.V + LT - 1) / LT;
  const long M = net_rows(h);
  const int mb = (int)((M + LT - 1) / LT);
  cudaStream_t s = h->stream;
  const int K = NT_TAP * kChan[l];
  const int co = kChan[l + 1];
  if (co == 32)
    count_launch(), k_wgrad<32><<<dim3(K, n->rb), LT, 0, s>>>(M, K, n->T[l], gout, n->rows_per_block, n->wpart);
  else
    count_launch(), k_wgrad<16><<<dim3(K, n->rb), LT, 0, s>>>(M, K, n->T[l], gout, n->rows_per_block, n->wpart);
  if (l > 0) {
    if (co == 32)
      count_launch(), k_mix_adj<32><<<mb, LT, 0, s>>>(M, K, gout, n->W[l], n->gT);
    else
      count_launch(), k_mix_adj<16><<<mb, LT, 0, s>>>(M, K, gout, n->W[l], n->gT);
    count_launch(), k_transport_adj<N><<<dim3(nb, kChan[l]), LT, 0, s>>>(
        g, (const float2*)h->U32, (const float2*)h->Uinv32, n->gT, kChan[l], gin);
  }
}

template <int N>
static void unembed_adj_n(susy_b200_net* n, double sc) {
  const Geo& g = n->h->g;
  const int nb = (g.V + LT - 1) / LT;
  count_launch(), k_unembed_adj<N><<<nb, LT, 0, n->h->stream>>>(g, (const float2*)n->h->U32,
                                                                 n->tfd, sc, n->gA);
}

// Loss of one pair (r, e = A^-1 r, A = D^dag D + fmass^2 + sigma):
//   sigma < 0:  |N(r) - e|^2 / |e|^2
//   sigma >= 0: (d, A d) / (e, A e) with d = N(r) - e and (e, A e) = Re<e, r>,
//               the A-norm error CG minimises
// grad (complex interleaved, the layout of set_weights) += dL/dW*
extern "C" int susy_b200_net_loss_grad2(susy_b200_net* n, const void* r, const void* e,
                                        double sigma, double* loss, double* grad) {
  if (!n || !r || !e || !loss) return SUSY_B200_EINVAL;
  susy_b200_lattice* h = n->h;
  cudaStream_t s = h->stream;
  // training differentiates the FP32 forward pass
  net_forward(n, r, n->tfz, false);
  const long nc = tf_complex(h);
  const int db = (int)((nc + 255) / 256);
  count_launch(), k_diff<<<db, 256, 0, s>>>(nc, n->tfz, (const double2*)e, n->tfd, n->part);
  std::vector<double> hp(2 * (size_t)db);
  cudaMemcpyAsync(hp.data(), n->part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (!ck(h, cudaStreamSynchronize(s))) return SUSY_B200_ECUDA;
  double d2 = 0.0, e2 = 0.0;
  for (int b = 0; b < db; b++) {
    d2 += hp[2 * b];
    e2 += hp[2 * b + 1];
  }
  if (!(e2 > 0.0)) return set_err(h, SUSY_B200_EINVAL);
  double scale = 1.0 / e2;
  *loss = d2 / e2;
  if (sigma >= 0.0) {
    // A d into tfz (the forward output is no longer needed)
    const double fm2 = h->prm.fmass > 1e-8 ? h->prm.fmass * h->prm.fmass : 0.0;
    void* t = scratch_tf(h, 0, 64);
    if (!t) return SUSY_B200_ENOMEM;
    dev_fop(h, n->tfd, t, 1, 64, nullptr, 0.0, nullptr, nullptr);
    dev_fop(h, t, n->tfz, -1, 64, n->tfd, fm2 + sigma, nullptr, nullptr);
    double* part = partials(h, 3);
    if (!part) return SUSY_B200_ENOMEM;
    const int nb = rdot_partials(nc, n->tfd, n->tfz, part, s);
    const double dad = host_sum(h, part, nb, 0);
    rdot_partials(nc, e, r, part, s);
    const double ear = host_sum(h, part, nb, 0);
    if (!(ear > 0.0)) return set_err(h, SUSY_B200_EINVAL);
    *loss = dad / ear;
    scale = 1.0 / ear;
    copy_field(nc, n->tfz, n->tfd, s);   // the gradient w.r.t. N(r)* is A d / (e, A e)
  }
  if (!grad) return SUSY_B200_OK;
  switch (h->N) {
    case 2: unembed_adj_n<2>(n, scale); break;
    case 3: unembed_adj_n<3>(n, scale); break;
    default: unembed_adj_n<4>(n, scale); break;
  }
  float2* gout = n->gA;
  float2* gin = n->gB;
  size_t off[3];
  off[0] = 0;
  off[1] = 2 * (size_t)net_kw(0);
  off[2] = off[1] + 2 * (size_t)net_kw(1);
  for (int l = 2; l >= 0; l--) {
    switch (h->N) {
      case 2: backward_layer<2>(n, l, gout, gin); break;
      case 3: backward_layer<3>(n, l, gout, gin); break;
      default: backward_layer<4>(n, l, gout, gin); break;
    }
    const int ci = kChan[l], co = kChan[l + 1];
    const int K = NT_TAP * ci;
    std::vector<double2> wp((size_t)n->rb * K * co);
    cudaMemcpyAsync(wp.data(), n->wpart, wp.size() * sizeof(double2), cudaMemcpyDeviceToHost, s);
    if (!ck(h, cudaStreamSynchronize(s))) return SUSY_B200_ECUDA;
    // partial[rb][k c_in][c_out] -> grad[k][c_out][c_in]
    for (int k = 0; k < NT_TAP; k++)
      for (int c = 0; c < ci; c++)
        for (int d = 0; d < co; d++) {
          double x = 0.0, y = 0.0;
          for (int b = 0; b < n->rb; b++) {
            const double2 v = wp[((size_t)b * K + (size_t)k * ci + c) * co + d];
            x += v.x;
            y += v.y;
          }
          const size_t dst = off[l] + 2 * (((size_t)k * co + d) * ci + c);
          grad[dst] += x;
          grad[dst + 1] += y;
        }
    std::swap(gout, gin);
  }
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

extern "C" int susy_b200_net_loss_grad(susy_b200_net* n, const void* r, const void* e,
                                       double* loss, double* grad) {
  return susy_b200_net_loss_grad2(n, r, e, -1.0, loss, grad);
}
