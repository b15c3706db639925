// The structured test meshes' geometric factors computed on the device
// (nkb_geom_fill_device): the same per-point arithmetic as the host fill
// (nkb_geom.h), one thread per element and quadrature point, so that a mesh
// of tens of thousands of curved elements needs neither the host loop nor
// the copy of its factors to the device. Device sin / cos may round the last
// bit differently from the host's.
#include "nkb_geom.h"
#include "nkb_internal.h"

#include <cuda_runtime.h>

#include <algorithm>

namespace nkb
{
namespace
{
constexpr int kGeomMaxPoints = 32;

struct GeomDev
{
    int shape, n, deformed, nq[3];
    double amp;
    double z[3][kGeomMaxPoints];
};

__global__ void k_geom_fill(GeomDev g, const int *__restrict__ cells, long nelmt, long nt, long ncol,
                            double *__restrict__ jac, double *__restrict__ df,
                            double *__restrict__ xyz)
{
    using namespace geom;
    const int epc = ElementsPerCell(g.shape);
    const long np = g.deformed || xyz ? nelmt * nt : nelmt;
    const long pe = g.deformed || xyz ? nt : 1; // threads per element
    for (long idx = blockIdx.x * long(blockDim.x) + threadIdx.x; idx < np;
         idx += long(gridDim.x) * blockDim.x)
    {
        const long e = idx / pe, q = idx % pe;
        const long c = e / epc;
        const int s = int(e % epc), cell = cells ? cells[c] : int(c);
        const Affine A = CellMap(g.shape, g.n, cell, s);
        const int i = int(q % g.nq[0]), j = int((q / g.nq[0]) % g.nq[1]),
                  k = int(q / (long(g.nq[0]) * g.nq[1]));
        double eta[3] = {g.z[0][i], g.z[1][j], g.z[2][k]};
        double xp[3], Ji[3][3], jv;
        if (g.deformed || q == 0)
        {
            double et[3] = {eta[0], eta[1], eta[2]};
            if (!g.deformed)
                et[0] = et[1] = et[2] = -0.5; // any interior point: affine
            AtPoint(g.shape, g.amp, A, et, jv, Ji, xp);
            const long col = g.deformed ? e * nt + q : e;
            jac[col]       = jv;
            for (int kk = 0; kk < 3; ++kk)
                for (int jj = 0; jj < 3; ++jj)
                    df[(kk * 3 + jj) * ncol + col] = Ji[jj][kk];
            if (xyz && g.deformed)
                for (int a = 0; a < 3; ++a)
                    xyz[a * nelmt * nt + e * nt + q] = xp[a];
        }
        if (xyz && !g.deformed)
        {
            AtPoint(g.shape, g.amp, A, eta, jv, Ji, xp);
            for (int a = 0; a < 3; ++a)
                xyz[a * nelmt * nt + e * nt + q] = xp[a];
        }
    }
}
} // namespace
} // namespace nkb

using namespace nkb;

extern "C" int nkb_geom_fill_device(const nkb_geom_request *req, double *jac, double *df,
                                    double *xyz, int device, void *stream)
{
    ClearError();
    if (!req || !jac || !df)
        return SetError(NKB_ERR_INVALID, "nkb_geom_fill_device: NULL argument");
    if (req->shape != NKB_HEX && req->shape != NKB_PRISM && req->shape != NKB_TET)
        return SetError(NKB_ERR_INVALID, "nkb_geom_fill_device: bad shape %d", req->shape);
    if (!req->deformed && req->amp != 0.0)
        return SetError(NKB_ERR_INVALID, "nkb_geom_fill_device: curved geometry must be deformed");
    GeomDev g;
    g.shape    = req->shape;
    g.n        = req->n;
    g.deformed = req->deformed ? 1 : 0;
    g.amp      = req->amp;
    for (int d = 0; d < 3; ++d)
    {
        if (!req->z[d] || req->nq[d] < 1 || req->nq[d] > kGeomMaxPoints)
            return SetError(NKB_ERR_INVALID, "nkb_geom_fill_device: points of dir %d (1..%d)", d,
                            kGeomMaxPoints);
        g.nq[d] = req->nq[d];
        for (int i = 0; i < req->nq[d]; ++i)
            g.z[d][i] = req->z[d][i];
    }
    const long ncells = req->ncells > 0 ? req->ncells : long(req->n) * req->n * req->n;
    if (req->n < 1 || (req->ncells > 0 && !req->cells))
        return SetError(NKB_ERR_INVALID, "nkb_geom_fill_device: bad cells");
    if (req->cells)
        for (long c = 0; c < ncells; ++c)
            if (req->cells[c] < 0 || long(req->cells[c]) >= long(req->n) * req->n * req->n)
                return SetError(NKB_ERR_INVALID, "nkb_geom_fill_device: cell %d outside the box",
                                req->cells[c]);
    const long nelmt = ncells * geom::ElementsPerCell(req->shape);
    const long nt    = long(g.nq[0]) * g.nq[1] * g.nq[2];
    const long ncol  = g.deformed ? nelmt * nt : nelmt;
    if (nelmt == 0)
        return NKB_OK;
    NKB_CUDA_TRY(cudaSetDevice(device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int *dcells    = nullptr;
    if (req->cells)
    {
        NKB_CUDA_TRY(cudaMalloc(&dcells, ncells * sizeof(int)));
        if (cudaMemcpyAsync(dcells, req->cells, ncells * sizeof(int), cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
        {
            cudaFree(dcells);
            return SetError(NKB_ERR_CUDA, "nkb_geom_fill_device: cells");
        }
    }
    const long np  = (g.deformed || xyz) ? nelmt * nt : nelmt;
    const int grid = int(std::max<long>(1, std::min<long>((np + 255) / 256, 148L * 16)));
    k_geom_fill<<<grid, 256, 0, s>>>(g, dcells, nelmt, nt, ncol, jac, df, xyz);
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess)
        ce = cudaStreamSynchronize(s);
    cudaFree(dcells);
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "nkb_geom_fill_device: %s", cudaGetErrorString(ce));
    return NKB_OK;
}
