// Instantiation of the tuned Hex Helmholtz kernels in FP64 (split from the
// other precision so the two compile in parallel).
#include "nkb_hex_kernel.cuh"

namespace nkb
{
template int HexLaunchT<double>(const nkb_op *, const HexArgs<double> &, bool, cudaStream_t, int, bool);
} // namespace nkb
