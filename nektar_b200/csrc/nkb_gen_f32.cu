// Compile-time-size Prism / Tet Helmholtz kernels, FP32 (nkb_generic_kernel.cuh).
#include "nkb_generic_kernel.cuh"

namespace nkb
{
template int LaunchHelmStatic<float>(const nkb_op *, const GenArgs<float> &, cudaStream_t);
} // namespace nkb
