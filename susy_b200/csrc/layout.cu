// Conversions between the reference's host layout and the device layout.
//
// Reference layout (4d_Q16/susy/lattice.h:18-59): an array over sites in
// node_index order (generic/layout_hyper_prime.c:157-170: even-parity sites
// first, lexicographic within each parity), each site holding K matrices
// e[N][N] of {double re, im}; a Twist_Fermion is K = 16
// {Fsite, Flink[5], Fplaq[10]}, link-type fields are K = 5.
// Device layout: structure of arrays, lexicographic sites (common.cuh).
#include "common.cuh"
#include "kernels.h"

namespace susy {

constexpr int LT = 256;

SUSY_D int node_index(const Geo& g, int s) {
  const Site c = site_of(g, s);
  return ((c.x + c.y + c.z + c.t) & 1) ? (s + g.V) / 2 : s / 2;
}

// aos: V sites x K x N x N complex (node_index order) -> soa (lexicographic)
template <typename T>
__global__ void k_aos_to_soa(Geo g, int K, int NN, const double2* aos, T* soa) {
  const long idx = (long)blockIdx.x * LT + threadIdx.x;
  const long per = (long)K * NN;
  if (idx >= per * g.V) return;
  const int s = (int)(idx / per);
  const int e = (int)(idx % per);
  const double2 v = aos[(long)node_index(g, s) * per + e];
  T o;
  o.x = v.x;
  o.y = v.y;
  soa[(long)e * g.S + s] = o;
}

template <typename T>
__global__ void k_soa_to_aos(Geo g, int K, int NN, const T* soa, double2* aos) {
  const long idx = (long)blockIdx.x * LT + threadIdx.x;
  const long per = (long)K * NN;
  if (idx >= per * g.V) return;
  const int s = (int)(idx / per);
  const int e = (int)(idx % per);
  const T v = soa[(long)e * g.S + s];
  aos[(long)node_index(g, s) * per + e] = make_double2(v.x, v.y);
}

// Precision change of an SoA field (nelem complex per site row, padded)
template <typename TI, typename TO>
__global__ void k_convert(long n, const TI* in, TO* out) {
  const long i = (long)blockIdx.x * LT + threadIdx.x;
  if (i >= n) return;
  TI v = in[i];
  TO o;
  o.x = v.x;
  o.y = v.y;
  out[i] = o;
}

static inline int nbl(long n) { return (int)((n + LT - 1) / LT); }

void aos_to_soa(const Geo& g, int K, int N, const void* aos, void* soa, int prec, cudaStream_t st) {
  const long n = (long)K * N * N * g.V;
  if (prec == 64)
    count_launch(), k_aos_to_soa<double2><<<nbl(n), LT, 0, st>>>(g, K, N * N, (const double2*)aos, (double2*)soa);
  else
    count_launch(), k_aos_to_soa<float2><<<nbl(n), LT, 0, st>>>(g, K, N * N, (const double2*)aos, (float2*)soa);
}

void soa_to_aos(const Geo& g, int K, int N, const void* soa, void* aos, int prec, cudaStream_t st) {
  const long n = (long)K * N * N * g.V;
  if (prec == 64)
    count_launch(), k_soa_to_aos<double2><<<nbl(n), LT, 0, st>>>(g, K, N * N, (const double2*)soa, (double2*)aos);
  else
    count_launch(), k_soa_to_aos<float2><<<nbl(n), LT, 0, st>>>(g, K, N * N, (const float2*)soa, (double2*)aos);
}

void convert_field(long ncomplex, const void* in, int prec_in, void* out, int prec_out,
                   cudaStream_t st) {
  if (prec_in == 64 && prec_out == 32)
    count_launch(), k_convert<double2, float2><<<nbl(ncomplex), LT, 0, st>>>(ncomplex, (const double2*)in, (float2*)out);
  else if (prec_in == 32 && prec_out == 64)
    count_launch(), k_convert<float2, double2><<<nbl(ncomplex), LT, 0, st>>>(ncomplex, (const float2*)in, (double2*)out);
  else if (prec_in == 64)
    cudaMemcpyAsync(out, in, ncomplex * sizeof(double2), cudaMemcpyDeviceToDevice, st);
  else
    cudaMemcpyAsync(out, in, ncomplex * sizeof(float2), cudaMemcpyDeviceToDevice, st);
}

}  // namespace susy
