// Shared device-side building blocks for the susy_b200 kernels.
//
// Field layout in HBM (structure of arrays, sites fastest):
//   a matrix field with K components stores element (k, i, j) of site s at
//   f[((k * N + i) * N + j) * S + s], one complex (double2 / float2) each,
//   S = site stride (volume rounded up to a multiple of 32).
//   Sites are lexicographic, s = x + nx * (y + ny * (z + nz * t)).
// A warp therefore reads 32 consecutive sites of one matrix element as one
// 512 B (FP64) or 256 B (FP32) coalesced transaction.
//   Twist_Fermion: K = 16 (0 = site eta, 1..5 = link psi_a,
//                  6..15 = plaquette chi_ab, a < b, reference plaq_index order)
//   links, momenta, forces, Uinv: K = 5;  Fmunu: K = 10;  DmuUmu: K = 1
//   plaquette determinants: complex pd[(a * 5 + b) * S + s]  (a != b)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define SUSY_HD __host__ __device__ __forceinline__
#define SUSY_D __device__ __forceinline__

namespace susy {

// Host-side count of kernel launches made by this library (every launch
// site is written as "count_launch(), kernel<<<...>>>(...)").
void count_launch();
void count_launches(long long n);
long long thread_launch_count();

constexpr int NUMLINK = 5;
constexpr int NPLAQ = 10;
constexpr int NTF = 16;

template <typename R> struct CT;
template <> struct CT<double> { typedef double2 T; };
template <> struct CT<float> { typedef float2 T; };

template <typename R>
struct Cx {
  R re, im;
  SUSY_HD Cx() {}
  SUSY_HD Cx(R r, R i) : re(r), im(i) {}
};

template <typename R> SUSY_HD Cx<R> operator+(Cx<R> a, Cx<R> b) { return Cx<R>(a.re + b.re, a.im + b.im); }
template <typename R> SUSY_HD Cx<R> operator-(Cx<R> a, Cx<R> b) { return Cx<R>(a.re - b.re, a.im - b.im); }
template <typename R> SUSY_HD Cx<R> operator*(Cx<R> a, Cx<R> b) {
  return Cx<R>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename R> SUSY_HD Cx<R> operator*(R s, Cx<R> a) { return Cx<R>(s * a.re, s * a.im); }
template <typename R> SUSY_HD Cx<R> conj(Cx<R> a) { return Cx<R>(a.re, -a.im); }

template <int N, typename R>
struct Mat {
  Cx<R> e[N][N];
  SUSY_HD void zero() {
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) e[i][j] = Cx<R>(0, 0);
  }
};

// ---------------------------------------------------------------------------
// Global-memory access
template <typename R>
SUSY_D Cx<R> ldc(const typename CT<R>::T* p) {
  typename CT<R>::T v = __ldg(p);
  return Cx<R>(v.x, v.y);
}

template <typename R>
SUSY_D void stc(typename CT<R>::T* p, Cx<R> c) {
  typename CT<R>::T v;
  v.x = c.re;
  v.y = c.im;
  *p = v;
}

// Load component k of a matrix field at site s (ADJ: load the adjoint)
template <int N, typename R, bool ADJ = false>
SUSY_D Mat<N, R> ldm(const typename CT<R>::T* f, int k, int s, int S) {
  Mat<N, R> m;
  const typename CT<R>::T* p = f + (size_t)(k * N * N) * S + s;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      Cx<R> v = ldc<R>(p + (size_t)(i * N + j) * S);
      if (ADJ)
        m.e[j][i] = conj(v);
      else
        m.e[i][j] = v;
    }
  return m;
}

template <int N, typename R>
SUSY_D void stm(typename CT<R>::T* f, int k, int s, int S, const Mat<N, R>& m) {
  typename CT<R>::T* p = f + (size_t)(k * N * N) * S + s;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) stc<R>(p + (size_t)(i * N + j) * S, m.e[i][j]);
}

// Trace of component k at site s (only the diagonal is read)
template <int N, typename R, bool ADJ = false>
SUSY_D Cx<R> ldtr(const typename CT<R>::T* f, int k, int s, int S) {
  const typename CT<R>::T* p = f + (size_t)(k * N * N) * S + s;
  Cx<R> t(0, 0);
#pragma unroll
  for (int i = 0; i < N; i++) t = t + ldc<R>(p + (size_t)(i * N + i) * S);
  return ADJ ? conj(t) : t;
}

// ---------------------------------------------------------------------------
// Matrix algebra in registers.  mode: 0 = A B, 1 = A B^dag, 2 = A^dag B
// acc += s * op(A) op(B): the right factor is scaled once (2 N^2 multiplies)
// and every complex multiply-add is four explicit fused multiply-adds into
// the accumulator (written as sums of products, the compiler would round
// each product and add separately).
template <int M, int N, typename R>
SUSY_D void mac(Mat<N, R>& acc, R s, const Mat<N, R>& A, const Mat<N, R>& B) {
  Cx<R> bs[N][N];
#pragma unroll
  for (int k = 0; k < N; k++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      const Cx<R> b = (M == 1) ? conj(B.e[j][k]) : B.e[k][j];
      bs[k][j] = Cx<R>(s * b.re, s * b.im);
    }
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int k = 0; k < N; k++) {
      const Cx<R> a = (M == 2) ? conj(A.e[k][i]) : A.e[i][k];
#pragma unroll
      for (int j = 0; j < N; j++) {
        R re = acc.e[i][j].re, im = acc.e[i][j].im;
        re = fma(a.re, bs[k][j].re, re);
        re = fma(-a.im, bs[k][j].im, re);
        im = fma(a.re, bs[k][j].im, im);
        im = fma(a.im, bs[k][j].re, im);
        acc.e[i][j] = Cx<R>(re, im);
      }
    }
}

// Matrix accumulator of the table-driven operator kernels
template <int N, typename R>
struct AccMat {
  Mat<N, R> m;
  SUSY_D void zero() { m.zero(); }
  SUSY_D void add(R s, const Mat<N, R>& A, const Mat<N, R>& B) { mac<0>(m, s, A, B); }
  SUSY_D Mat<N, R> get() const { return m; }
};

template <int N, typename R>
SUSY_D void axpy(Mat<N, R>& acc, Cx<R> c, const Mat<N, R>& A) {
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) acc.e[i][j] = acc.e[i][j] + c * A.e[i][j];
}

template <int N, typename R>
SUSY_D Mat<N, R> mul(const Mat<N, R>& A, const Mat<N, R>& B) {
  Mat<N, R> c;
  c.zero();
  mac<0>(c, (R)1, A, B);
  return c;
}

template <int N, typename R>
SUSY_D Mat<N, R> adjm(const Mat<N, R>& A) {
  Mat<N, R> c;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) c.e[i][j] = conj(A.e[j][i]);
  return c;
}

template <int N, typename R>
SUSY_D Cx<R> trace(const Mat<N, R>& A) {
  Cx<R> t(0, 0);
#pragma unroll
  for (int i = 0; i < N; i++) t = t + A.e[i][i];
  return t;
}

// Tr(A B)
template <int N, typename R>
SUSY_D Cx<R> trace_nn(const Mat<N, R>& A, const Mat<N, R>& B) {
  Cx<R> t(0, 0);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int k = 0; k < N; k++) t = t + A.e[i][k] * B.e[k][i];
  return t;
}

// Re Tr(A^dag B)
template <int N, typename R>
SUSY_D double rdot(const Mat<N, R>& A, const Mat<N, R>& B) {
  double t = 0;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++)
      t += (double)A.e[i][j].re * B.e[i][j].re + (double)A.e[i][j].im * B.e[i][j].im;
  return t;
}

// ---------------------------------------------------------------------------
// Geometry.  Link offsets e_0..e_3 are the axes, e_4 = (-1,-1,-1,-1).
struct Geo {
  int nx, ny, nz, nt;
  int V;    // sites
  int S;    // site stride of every field
  int pbc;  // temporal fermion boundary condition, +1 or -1
};

struct Site {
  int x, y, z, t, s;
};

SUSY_D Site site_of(const Geo& g, int s) {
  Site c;
  c.s = s;
  c.x = s % g.nx;
  int r = s / g.nx;
  c.y = r % g.ny;
  r /= g.ny;
  c.z = r % g.nz;
  c.t = r / g.nz;
  return c;
}

SUSY_D int wrap(int v, int n) {
  v -= (v >= n) ? n : 0;
  v -= (v >= n) ? n : 0;
  v += (v < 0) ? n : 0;
  v += (v < 0) ? n : 0;
  return v;
}

// Net displacement of a sum of link offsets, packed as a compile-time int
// per axis: each link index a in [0,5) contributes e_a.
SUSY_HD constexpr int ex(int a) { return a == 0 ? 1 : (a == 4 ? -1 : 0); }
SUSY_HD constexpr int ey(int a) { return a == 1 ? 1 : (a == 4 ? -1 : 0); }
SUSY_HD constexpr int ez(int a) { return a == 2 ? 1 : (a == 4 ? -1 : 0); }
SUSY_HD constexpr int et(int a) { return a == 3 ? 1 : (a == 4 ? -1 : 0); }

// Index of x + d (|d| per axis <= 3)
SUSY_D int nbr(const Geo& g, const Site& c, int dx, int dy, int dz, int dt) {
  int x = wrap(c.x + dx, g.nx), y = wrap(c.y + dy, g.ny);
  int z = wrap(c.z + dz, g.nz), t = wrap(c.t + dt, g.nt);
  return x + g.nx * (y + g.ny * (z + g.nz * t));
}

// Temporal BC factor of a path with net time displacement dt starting at c
// (reference setup_offset.c:67-145: PBC when t + dt leaves [0, nt-1])
template <typename R>
SUSY_D R bcf(const Geo& g, const Site& c, int dt) {
  int t = c.t + dt;
  return (t < 0 || t > g.nt - 1) ? (R)g.pbc : (R)1;
}

// plaq_index for a < b (reference setup_lambda.c:142-152)
SUSY_HD constexpr int pidx(int a, int b) {
  return a < b ? (a * 4 - a * (a + 1) / 2 + b - 1) : (b * 4 - b * (b + 1) / 2 + a - 1);
}

// Sign of the permutation (a,b,c,d,e) of (0..4); 0 if not a permutation
SUSY_HD constexpr int eps5(int a, int b, int c, int d, int e) {
  int v[5] = {a, b, c, d, e};
  int sgn = 1;
  for (int i = 0; i < 5; i++)
    for (int j = i + 1; j < 5; j++) {
      if (v[i] == v[j]) return 0;
      if (v[i] > v[j]) sgn = -sgn;
    }
  return sgn;
}

}  // namespace susy

namespace susy {
// Deterministic block-wide FP64 sum; result valid on thread 0 only.
template <int NT>
SUSY_D double block_sum(double v) {
  __shared__ double sh[NT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < NT / 32; i++) r += sh[i];
  return r;
}
}  // namespace susy
