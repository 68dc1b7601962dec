// Host-side launch interface of the susy_b200 kernels (internal C++ API).
// All launches are asynchronous on the given stream; fields are in the
// device layout described in common.cuh.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"

namespace susy {

constexpr int MS_MAXS = 32;

// Device-resident state of one multi-shift solve (FP64 scalars)
struct MsState {
  double rsq, rsqstop, source_norm, cd;
  int iter, maxcg, nshift, skip, skip_b, pad;
  double shift[MS_MAXS];
  double zeta_i[MS_MAXS], zeta_im1[MS_MAXS], zeta_ip1[MS_MAXS];
  double beta_i[MS_MAXS], beta_im1[MS_MAXS], alpha[MS_MAXS];
  int converged[MS_MAXS], active_p[MS_MAXS];
};

struct MsVecs {
  void* p[MS_MAXS];    // p[0] = p0 (the DSq input), p[j] for shifts j >= 1
  void* psi[MS_MAXS];  // solutions
  void* r;
  void* mp;
};

// fermion_op.cu
template <typename R>
void fermion_op(const Geo& g, int N, const void* U, const void* Uinv, const void* pd,
                const void* src, void* dst, int sign, double G, const void* add, double addc,
                double* dot, const int* skip, cudaStream_t st);
int fop_partials(const Geo& g);

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
             double errormin, cudaStream_t s);
void ms_scalars1(MsState* st, const double* part, int np, cudaStream_t s);
void ms_scalars2(MsState* st, const double* part, int np, cudaStream_t s);
void ms_update_a(MsState* st, const MsVecs& v, int prec, long n, double* part, cudaStream_t s);
void ms_update_b(MsState* st, const MsVecs& v, int prec, long n, cudaStream_t s);
void norm2_partials(const void* x, int prec, long n, double* part, cudaStream_t s);

}  // namespace susy
