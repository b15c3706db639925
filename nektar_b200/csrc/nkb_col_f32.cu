// Prism / Tet column Helmholtz kernels, FP32 (nkb_col_kernel.cuh).
#include "nkb_col_kernel.cuh"

namespace nkb
{
template int LaunchColHelm<float>(const nkb_op *, const GenArgs<float> &, cudaStream_t);
} // namespace nkb
