// Internal declarations shared by the trajectory driver and the solvers.
#pragma once
#include "lattice.h"

namespace susy {
void node_prn_init(HostPrn& p, int seed, int index);
double node_myrand(HostPrn& p);
double host_sum(susy_b200_lattice* h, const double* dpart, int n, int offset);
int multishift_mixed(susy_b200_lattice* h, const void* src, void* const* psim, int norder,
                     const double* shift, int MaxCG, double errormin, double* size_r, int* iters);
}  // namespace susy
