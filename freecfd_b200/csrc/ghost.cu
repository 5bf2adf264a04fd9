// Ghost-state update compiled without multiply-add contraction (-fmad=false):
// every operation of the boundary-condition formulas rounds once, as in the
// reference, so ghost values that feed the bit-exact LSQ gradients are the
// reference's doubles (up to CUDA pow vs libm pow in the BC branches that
// call pow).
#include "kernels.cuh"

namespace fcfd {
template __global__ void k_ghost_minmax<double>(DevCase, DevMesh, double *, unsigned long long *, int *);
template __global__ void k_ghost_minmax<Dual<double>>(DevCase, DevMesh, Dual<double> *, unsigned long long *, int *);
template __global__ void k_ghost_minmax<Dual<float>>(DevCase, DevMesh, Dual<float> *, unsigned long long *, int *);
}  // namespace fcfd
