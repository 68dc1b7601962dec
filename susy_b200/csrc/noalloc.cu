// D^dag D (+ fmass^2) on caller-owned device fields with no device
// allocation at all (susy_b200_DSq_noalloc, include/susy_b200.h).
//
// The regular DSq entry points keep their intermediate field D src in
// memory the lattice handle allocates on first use.  This variant puts that
// intermediate field in a fixed file-scope device array instead, so a
// caller that owns every device buffer itself (and has no handle) can apply
// the operator without this library ever calling cudaMalloc.  The array is
// part of the loaded module: every GPU that loads the library holds its
// 16 MiB until the process exits.
#include "../../include/susy_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace susy {

// Capacity of the intermediate field in complex doubles: 16 NCOL^2 S <= 2^20
// (16 MiB), e.g. 8^4 sites for NCOL = 2, 3 or 4.
constexpr long NOALLOC_MAX_COMPLEX = 1L << 20;

static __device__ __align__(256) double2 g_noalloc_tmp[NOALLOC_MAX_COMPLEX];

// Device address of g_noalloc_tmp on the current device.  In host code the
// array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress with the device current.  It is looked up on every
// call rather than cached: after a cudaDeviceReset the module is loaded
// again, possibly at another address, and a cached pointer would be stale.
// Once the module is loaded the lookup is a table search in the runtime.
static int noalloc_scratch(void** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_tmp) != cudaSuccess || !p) {
    cudaGetLastError();
    return SUSY_B200_ECUDA;
  }
  *out = p;
  return SUSY_B200_OK;
}

}  // namespace susy

using namespace susy;

extern "C" int susy_b200_DSq_noalloc(int nx, int ny, int nz, int nt, int ncol, int pbc, double G,
                                     double fmass, const void* links, const void* Uinv,
                                     const void* plaqdet, const void* src, void* dst,
                                     void* cuda_stream) {
  // Extents are checked and the volume formed in 64 bits before anything is
  // sized from it: a volume that wrapped in int could pass the scratch bound
  // while the kernels index the caller's fields with the real extents.
  Geo g;
  if (!make_geo(nx, ny, nz, nt, ncol, pbc, &g)) {
    const bool shape_ok = ncol >= 2 && ncol <= 4 && nx >= 2 && ny >= 2 && nz >= 2 && nt >= 2 &&
                          !((nx | ny | nz | nt) & 1) && (pbc == 1 || pbc == -1);
    // well-formed extents whose volume is only too large: the scratch limit
    return shape_ok ? SUSY_B200_ESCRATCH : SUSY_B200_EINVAL;
  }
  if ((long)NTF * ncol * ncol * g.S > NOALLOC_MAX_COMPLEX) return SUSY_B200_ESCRATCH;
  const bool doG = G > 1e-8;
  if (!links || !src || !dst || (doG && (!Uinv || !plaqdet))) return SUSY_B200_EINVAL;
  void* tmp = nullptr;
  int rc = noalloc_scratch(&tmp);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)cuda_stream;
  const double fm2 = fmass > 1e-8 ? fmass * fmass : 0.0;
  // The first application writes every entry the second one reads, so the
  // shared array needs no clearing between calls.
  fermion_op<double>(g, ncol, links, Uinv, plaqdet, src, tmp, 1, G, nullptr, 0.0, nullptr,
                     nullptr, FOP_MAT_CM, nullptr, st);
  fermion_op<double>(g, ncol, links, Uinv, plaqdet, tmp, dst, -1, G, fm2 != 0.0 ? src : nullptr,
                     fm2, nullptr, nullptr, FOP_MAT_CM, nullptr, st);
  if (cudaGetLastError() != cudaSuccess) return SUSY_B200_ECUDA;
  return SUSY_B200_OK;
}
