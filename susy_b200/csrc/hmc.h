// Internal declarations shared by the trajectory driver and the solvers.
#pragma once
#include "lattice.h"

namespace susy {
void node_prn_init(HostPrn& p, int seed, int index);
double node_myrand(HostPrn& p);
double host_sum(susy_b200_lattice* h, const double* dpart, int n, int offset);
// on_frozen as for multishift_fp64; redo[j] (norder entries, if given) is
// set for every shift whose solution changed after on_frozen(j) was called
// (a per-shift correction, or the FP64 fallback)
int multishift_mixed(susy_b200_lattice* h, const void* src, void* const* psim, int norder,
                     const double* shift, int MaxCG, double errormin, double* size_r, int* iters,
                     const FrozenHook* on_frozen = nullptr, char* redo = nullptr);
}  // namespace susy
