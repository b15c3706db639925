// Internal declarations shared by the host and CUDA translation units of
// libnekb200.so. Not part of the C ABI (include/nektar_b200.h is).
#pragma once

#include "../../include/nektar_b200.h"

#include <cstdarg>
#include <cstddef>
#include <cstdio>

namespace nkb
{

// Records the message for nkb_last_error() (thread local) and returns code.
int SetError(int code, const char *fmt, ...);
void ClearError();

// Number of coefficients of a 3-D element (ShapeType.hpp:214-225, 366-374).
inline int NumCoeffs(int shape, int nm)
{
    if (shape == NKB_HEX)
        return nm * nm * nm;
    if (shape == NKB_PRISM)
        return nm * nm * (nm + 1) / 2;
    return nm * (nm + 1) * (nm + 2) / 6;
}

// Tabulated modes of the 1-D table in direction d (Modified_A/B/C).
inline int TableModes(int shape, int d, int nm)
{
    int bt = 0;
    if (shape == NKB_PRISM)
        bt = (d == 2) ? 1 : 0;
    else if (shape == NKB_TET)
        bt = d;
    if (bt == 0)
        return nm;
    if (bt == 1)
        return nm * (nm + 1) / 2;
    return nm * (nm + 1) * (nm + 2) / 6;
}

// Radau weight factor of MatrixFree SetUpZW (Operator.hpp:592-625).
inline double WeightFactor(int ptype)
{
    if (ptype == NKB_RADAU_A1)
        return 0.5;
    if (ptype == NKB_RADAU_A2)
        return 0.25;
    return 1.0;
}

} // namespace nkb

#define NKB_CUDA_TRY(call)                                                                        \
    do                                                                                            \
    {                                                                                             \
        cudaError_t _e = (call);                                                                  \
        if (_e != cudaSuccess)                                                                    \
            return ::nkb::SetError(NKB_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,       \
                                   cudaGetErrorString(_e));                                       \
    } while (0)
