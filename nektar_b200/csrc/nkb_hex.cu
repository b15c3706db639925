// Kernel selection for the element operators. Tuned Hex kernels are chosen
// here when one is compiled for the operator's (nm, nq, precision); every
// other operator runs the shape-generic kernels of nkb_ops.cu.
#include "nkb_op.h"

namespace nkb
{

int ChooseKernel(nkb_op *op)
{
    op->variant = 0;
    const int eb = op->precision == NKB_FP64 ? 8 : 4;
    if (GenericSmemBytes(op, eb) > 200 * 1024)
        return SetError(NKB_ERR_UNSUPPORTED,
                        "nkb_op_create: nm=%d nq=(%d,%d,%d) needs %zu bytes of shared memory per "
                        "element", op->nm, op->nq[0], op->nq[1], op->nq[2], GenericSmemBytes(op, eb));
    return NKB_OK;
}

void FreeKernelData(nkb_op *op)
{
    op->kdata = nullptr;
}

template <typename T>
int LaunchOp(const nkb_op *op, const T *in, T *o0, T *o1, T *o2, const int *gmap,
             const double *gsign, cudaStream_t s)
{
    return LaunchGeneric<T>(op, in, o0, o1, o2, gmap, gsign, s);
}

template int LaunchOp<double>(const nkb_op *, const double *, double *, double *, double *,
                              const int *, const double *, cudaStream_t);
template int LaunchOp<float>(const nkb_op *, const float *, float *, float *, float *,
                             const int *, const double *, cudaStream_t);

} // namespace nkb
