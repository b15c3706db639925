// Instantiation of the tuned Hex Helmholtz kernels in FP32 (split from the
// other precision so the two compile in parallel).
#include "nkb_hex_kernel.cuh"

namespace nkb
{
template int HexLaunchT<float>(const nkb_op *, const HexArgs<float> &, bool, cudaStream_t, int, bool);
} // namespace nkb
