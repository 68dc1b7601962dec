// Fields derived from the links after every link update
// (reference update_o.c:31-34):
//   link determinants and inverses   compute_Uinv      utilities.c:117-127
//                                    find_det / invert determinant.c:10-85
//   plaquette determinants, ZW*      compute_plaqdet   utilities.c:17-110
//   DmuUmu                           compute_DmuUmu    action.c:15-62
//   Fmunu                            compute_Fmunu     action.c:71-98
// Determinant and inverse use Gauss-Jordan elimination with partial pivoting
// on |re| + |im| (LAPACK's pivot measure) in registers, for any NCOL <= 4,
// in place of the reference's LAPACK zgetrf/zgetri calls.
#include "common.cuh"
#include "kernels.h"
#include "linalg.cuh"

namespace susy {

constexpr int DT = 128;

// det U_a(x) and U_a(x)^{-1} for every (site, link)
template <int N>
__global__ void k_det_inv(Geo g, const double2* U, double2* det, double2* Uinv) {
  const int idx = blockIdx.x * DT + threadIdx.x;
  if (idx >= g.V * NUMLINK) return;
  const int a = idx / g.V, s = idx % g.V;
  Mat<N, double> u = ldm<N, double>(U, a, s, g.S), ui;
  Cx<double> d;
  det_inv<N>(u, d, ui);
  stc<double>(det + (size_t)a * g.S + s, d);
  stm<N, double>(Uinv, a, s, g.S, ui);
}

// plaqdet[a][b] = conj(det U_a(x)) det U_b(x) conj(det U_b(x+a)) det U_a(x+b)
// and ZW*[a][b] = plaqdet (plaqdet - 1)^*   (utilities.c:80-96)
__global__ void k_plaqdet(Geo g, const double2* det, double2* pd, double2* zw) {
  const int s = blockIdx.x * DT + threadIdx.x;
  if (s >= g.V) return;
  Site c = site_of(g, s);
  Cx<double> d0[NUMLINK];
#pragma unroll
  for (int a = 0; a < NUMLINK; a++) d0[a] = ldc<double>(det + (size_t)a * g.S + s);
#pragma unroll
  for (int a = 0; a < NUMLINK; a++) {
    const int pa = nbr(g, c, ex(a), ey(a), ez(a), et(a));
#pragma unroll
    for (int b = 0; b < NUMLINK; b++) {
      if (a == b) continue;
      const int pb = nbr(g, c, ex(b), ey(b), ez(b), et(b));
      Cx<double> p = conj(d0[a]) * d0[b];
      p = p * conj(ldc<double>(det + (size_t)b * g.S + pa));
      p = ldc<double>(det + (size_t)a * g.S + pb) * p;
      stc<double>(pd + (size_t)(a * 5 + b) * g.S + s, p);
      stc<double>(zw + (size_t)(a * 5 + b) * g.S + s, p * conj(Cx<double>(p.re - 1.0, p.im)));
    }
  }
}

// DmuUmu = sum_a [U_a U_a^dag - (U_a^dag U_a)(x - a)] + G sum_{a!=b} (plaqdet - 1) I
template <int N>
__global__ void k_dmuumu(Geo g, const double2* U, const double2* pd, double G, int doG,
                         double2* D) {
  const int s = blockIdx.x * DT + threadIdx.x;
  if (s >= g.V) return;
  Site c = site_of(g, s);
  Mat<N, double> acc;
  acc.zero();
#pragma unroll
  for (int a = 0; a < NUMLINK; a++) {
    Mat<N, double> u = ldm<N, double>(U, a, s, g.S);
    mac<1>(acc, 1.0, u, u);
    Mat<N, double> um = ldm<N, double>(U, a, nbr(g, c, -ex(a), -ey(a), -ez(a), -et(a)), g.S);
    mac<2>(acc, -1.0, um, um);
  }
  if (doG) {
    Cx<double> t(0, 0);
#pragma unroll
    for (int a = 0; a < NUMLINK; a++)
#pragma unroll
      for (int b = 0; b < NUMLINK; b++) {
        if (a == b) continue;
        Cx<double> p = ldc<double>(pd + (size_t)(a * 5 + b) * g.S + s);
        t = t + G * Cx<double>(p.re - 1.0, p.im);
      }
#pragma unroll
    for (int i = 0; i < N; i++) acc.e[i][i] = acc.e[i][i] + t;
  }
  stm<N, double>(D, 0, s, g.S, acc);
}

// Fmunu[ab] = U_a U_b(x + a) - U_b U_a(x + b), a < b
template <int N>
__global__ void k_fmunu(Geo g, const double2* U, double2* F) {
  const int idx = blockIdx.x * DT + threadIdx.x;
  if (idx >= g.V * NPLAQ) return;
  const int p = idx / g.V, s = idx % g.V;
  Site c = site_of(g, s);
  int a = 0, b = 1;
  for (int aa = 0, k = 0; aa < NUMLINK; aa++)
    for (int bb = aa + 1; bb < NUMLINK; bb++, k++)
      if (k == p) { a = aa; b = bb; }
  const int pa = nbr(g, c, ex(a), ey(a), ez(a), et(a));
  const int pb = nbr(g, c, ex(b), ey(b), ez(b), et(b));
  Mat<N, double> acc;
  acc.zero();
  mac<0>(acc, 1.0, ldm<N, double>(U, a, s, g.S), ldm<N, double>(U, b, pa, g.S));
  mac<0>(acc, -1.0, ldm<N, double>(U, b, s, g.S), ldm<N, double>(U, a, pb, g.S));
  stm<N, double>(F, p, s, g.S, acc);
}

static inline int nb(long n) { return (int)((n + DT - 1) / DT); }

void compute_uinv(const Geo& g, int N, const void* U, void* det, void* Uinv, cudaStream_t st) {
  const long n = (long)g.V * NUMLINK;
  switch (N) {
    case 2: count_launch(), k_det_inv<2><<<nb(n), DT, 0, st>>>(g, (const double2*)U, (double2*)det, (double2*)Uinv); break;
    case 3: count_launch(), k_det_inv<3><<<nb(n), DT, 0, st>>>(g, (const double2*)U, (double2*)det, (double2*)Uinv); break;
    case 4: count_launch(), k_det_inv<4><<<nb(n), DT, 0, st>>>(g, (const double2*)U, (double2*)det, (double2*)Uinv); break;
  }
}

void compute_plaqdet(const Geo& g, const void* det, void* pd, void* zw, cudaStream_t st) {
  count_launch(), k_plaqdet<<<nb(g.V), DT, 0, st>>>(g, (const double2*)det, (double2*)pd, (double2*)zw);
}

void compute_dmuumu(const Geo& g, int N, const void* U, const void* pd, double G, void* D,
                    cudaStream_t st) {
  const int doG = G > 1e-8;
  switch (N) {
    case 2: count_launch(), k_dmuumu<2><<<nb(g.V), DT, 0, st>>>(g, (const double2*)U, (const double2*)pd, G, doG, (double2*)D); break;
    case 3: count_launch(), k_dmuumu<3><<<nb(g.V), DT, 0, st>>>(g, (const double2*)U, (const double2*)pd, G, doG, (double2*)D); break;
    case 4: count_launch(), k_dmuumu<4><<<nb(g.V), DT, 0, st>>>(g, (const double2*)U, (const double2*)pd, G, doG, (double2*)D); break;
  }
}

void compute_fmunu(const Geo& g, int N, const void* U, void* F, cudaStream_t st) {
  const long n = (long)g.V * NPLAQ;
  switch (N) {
    case 2: count_launch(), k_fmunu<2><<<nb(n), DT, 0, st>>>(g, (const double2*)U, (double2*)F); break;
    case 3: count_launch(), k_fmunu<3><<<nb(n), DT, 0, st>>>(g, (const double2*)U, (double2*)F); break;
    case 4: count_launch(), k_fmunu<4><<<nb(n), DT, 0, st>>>(g, (const double2*)U, (double2*)F); break;
  }
}

}  // namespace susy
