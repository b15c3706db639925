// Compile-time-size Prism / Tet Helmholtz kernels, FP64 (nkb_generic_kernel.cuh).
#include "nkb_generic_kernel.cuh"

namespace nkb
{
template int LaunchHelmStatic<double>(const nkb_op *, const GenArgs<double> &, cudaStream_t);
} // namespace nkb
