// Prism / Tet column Helmholtz kernels, FP64 (nkb_col_kernel.cuh).
#include "nkb_col_kernel.cuh"

namespace nkb
{
template int LaunchColHelm<double>(const nkb_op *, const GenArgs<double> &, cudaStream_t);
} // namespace nkb
