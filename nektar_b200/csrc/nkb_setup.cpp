// FP64 host-side setup of the B200 matrix-free path: 1-D quadrature and
// modified-basis tables, analytic geometric factors of the structured test
// meshes and the C0 assembly map of a hex box.
//
// The tables restate the published definitions the reference implements in
// LibUtilities/Foundations (GaussPoints.cpp:79-240, Basis.cpp:466-644) and
// LibUtilities/Polylib (Polylib.cpp: Gauss-Jacobi zeros by Newton iteration
// with deflation, Gauss-Lobatto / Gauss-Radau weights); the derivative matrix
// is formed from barycentric weights rather than Polylib's closed forms.
// Geometry follows GeomFactors::ComputeJac / ComputeDerivFactors
// (GeomFactors.cpp:248-477): jac = |det dx/dxi|, df[k*3+j] = d xi_j / d x_k,
// evaluated from the analytic Jacobian of the curved map.
#include "nkb_internal.h"
#include "nkb_geom.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace nkb
{

// Jacobi polynomial P_n^{a,b} and its derivative at z (three-term recurrence).
static void Jacobi(int n, double a, double b, double z, double *p, double *dp)
{
    double p0 = 1.0, p1 = 0.5 * (a - b + (a + b + 2.0) * z);
    double d0 = 0.0, d1 = 0.5 * (a + b + 2.0);
    if (n == 0)
    {
        *p = p0;
        if (dp)
            *dp = d0;
        return;
    }
    for (int k = 2; k <= n; ++k)
    {
        double c  = 2.0 * k + a + b;
        double a1 = 2.0 * k * (k + a + b) * (c - 2.0);
        double a2 = (c - 1.0) * (a * a - b * b);
        double a3 = (c - 2.0) * (c - 1.0) * c;
        double a4 = 2.0 * (k + a - 1.0) * (k + b - 1.0) * c;
        double pn = ((a2 + a3 * z) * p1 - a4 * p0) / a1;
        double dn = ((a2 + a3 * z) * d1 + a3 * p1 - a4 * d0) / a1;
        p0 = p1;
        p1 = pn;
        d0 = d1;
        d1 = dn;
    }
    *p = p1;
    if (dp)
        *dp = d1;
}

// n zeros of P_n^{a,b} in ascending order: Newton iteration with deflation of
// the zeros already found, started from Chebyshev-Gauss points.
static void JacobiZeros(int n, double a, double b, double *z)
{
    for (int k = 0; k < n; ++k)
    {
        double r = -std::cos((2.0 * k + 1.0) * M_PI / (2.0 * n));
        if (k > 0)
            r = 0.5 * (r + z[k - 1]);
        for (int it = 0; it < 100; ++it)
        {
            double p, dp;
            Jacobi(n, a, b, r, &p, &dp);
            double s = 0.0;
            for (int i = 0; i < k; ++i)
                s += 1.0 / (r - z[i]);
            double dr = -p / (dp - s * p);
            r += dr;
            if (std::fabs(dr) < 1e-15)
                break;
        }
        z[k] = r;
    }
}

static void BarycentricD(int np, const double *z, double *D)
{
    std::vector<double> lam(np, 1.0);
    for (int j = 0; j < np; ++j)
        for (int k = 0; k < np; ++k)
            if (k != j)
                lam[j] *= (z[j] - z[k]);
    for (int j = 0; j < np; ++j)
        lam[j] = 1.0 / lam[j];
    // D_ij = l_j'(z_i), stored column-major: D[j*np + i]
    for (int i = 0; i < np; ++i)
    {
        double diag = 0.0;
        for (int j = 0; j < np; ++j)
        {
            if (i == j)
                continue;
            double v                      = (lam[j] / lam[i]) / (z[i] - z[j]);
            D[std::size_t(j) * np + i]    = v;
            diag -= v;
        }
        D[std::size_t(i) * np + i] = diag;
    }
}

} // namespace nkb

using namespace nkb;

extern "C" int nkb_points(int ptype, int np, double *z, double *w, double *D)
{
    if (np < 2 || np > 64 || !z || !w)
        return SetError(NKB_ERR_INVALID, "nkb_points: bad size or NULL output");
    if (ptype == NKB_GLL)
    {
        // z: -1, zeros of P^{1,1}_{np-2}, 1; w_i = 2 / (np (np-1) P_{np-1}(z_i)^2)
        z[0]      = -1.0;
        z[np - 1] = 1.0;
        JacobiZeros(np - 2, 1.0, 1.0, z + 1);
        for (int i = 0; i < np; ++i)
        {
            double p;
            Jacobi(np - 1, 0.0, 0.0, z[i], &p, nullptr);
            w[i] = 2.0 / (double(np) * (np - 1) * p * p);
        }
    }
    else if (ptype == NKB_RADAU_A1 || ptype == NKB_RADAU_A2)
    {
        // Gauss-Radau-Jacobi with the end point -1 for weight (1-z)^a:
        // z: -1 and the zeros of P^{a,1}_{np-1};
        // w_i = C (1 - z_i) / P^{a,0}_{np-1}(z_i)^2, w_0 scaled by (b+1) = 1,
        // C = 2^a G(np+a) G(np) / (G(np) G(np+1+a) np)
        const double a = (ptype == NKB_RADAU_A1) ? 1.0 : 2.0;
        z[0]           = -1.0;
        JacobiZeros(np - 1, a, 1.0, z + 1);
        const double C = std::pow(2.0, a) * std::tgamma(np + a) / std::tgamma(np + 1.0 + a) /
                         double(np);
        for (int i = 0; i < np; ++i)
        {
            double p;
            Jacobi(np - 1, a, 0.0, z[i], &p, nullptr);
            w[i] = C * (1.0 - z[i]) / (p * p);
        }
    }
    else
    {
        return SetError(NKB_ERR_UNSUPPORTED, "nkb_points: points type %d not supported", ptype);
    }
    if (D)
        BarycentricD(np, z, D);
    return NKB_OK;
}

extern "C" int nkb_basis(int btype, int nm, int np, const double *z, const double *D,
                         double *bdata, double *dbdata)
{
    if (nm < 2 || nm > 32 || np < 2 || !z || !bdata)
        return SetError(NKB_ERR_INVALID, "nkb_basis: bad arguments");
    // Modified_B rows: (p, q) with q fastest, q < nm - p:
    //   p = 0: (1-z)/2, (1+z)/2, then (1-z)/2 (1+z)/2 P^{1,1}_{q-2}
    //   p = 1: (1-z)/2, then (1-z)/2 (1+z)/2 P^{1,1}_{q-2}
    //   p >= 2: ((1-z)/2)^p, then ((1-z)/2)^p (1+z)/2 P^{2p-1,1}_{q-1}
    // Modified_A is the p = 0 row; Modified_C repeats Modified_B row p+q for
    // every (p, q) with r < nm - p - q.
    auto modB = [&](int p, int q, double x) {
        double lo = 0.5 * (1.0 - x), hi = 0.5 * (1.0 + x), j;
        if (p == 0)
        {
            if (q == 0)
                return lo;
            if (q == 1)
                return hi;
            Jacobi(q - 2, 1.0, 1.0, x, &j, nullptr);
            return lo * hi * j;
        }
        if (p == 1)
        {
            if (q == 0)
                return lo;
            Jacobi(q - 1, 1.0, 1.0, x, &j, nullptr);
            return lo * hi * j;
        }
        double lp = std::pow(lo, p);
        if (q == 0)
            return lp;
        Jacobi(q - 1, 2.0 * p - 1.0, 1.0, x, &j, nullptr);
        return lp * hi * j;
    };
    std::size_t nb = 0;
    if (btype == NKB_MODIFIED_A)
    {
        for (int p = 0; p < nm; ++p, ++nb)
            for (int i = 0; i < np; ++i)
                bdata[nb * np + i] = modB(0, p, z[i]);
    }
    else if (btype == NKB_MODIFIED_B)
    {
        for (int p = 0; p < nm; ++p)
            for (int q = 0; q < nm - p; ++q, ++nb)
                for (int i = 0; i < np; ++i)
                    bdata[nb * np + i] = modB(p, q, z[i]);
    }
    else if (btype == NKB_MODIFIED_C)
    {
        for (int p = 0; p < nm; ++p)
            for (int q = 0; q < nm - p; ++q)
                for (int r = 0; r < nm - p - q; ++r, ++nb)
                    for (int i = 0; i < np; ++i)
                        bdata[nb * np + i] = modB(p + q, r, z[i]);
    }
    else
    {
        return SetError(NKB_ERR_UNSUPPORTED, "nkb_basis: basis type %d not supported", btype);
    }
    if (dbdata)
    {
        if (!D)
            return SetError(NKB_ERR_INVALID, "nkb_basis: dbdata needs D");
        for (std::size_t m = 0; m < nb; ++m)
            for (int i = 0; i < np; ++i)
            {
                double s = 0.0;
                for (int k = 0; k < np; ++k)
                    s += D[std::size_t(k) * np + i] * bdata[m * np + k];
                dbdata[m * np + i] = s;
            }
    }
    return int(nb);
}

// ---------------------------------------------------------------------------
// Structured test meshes
// ---------------------------------------------------------------------------
using namespace nkb::geom;

extern "C" long nkb_geom_nelmt(const nkb_geom_request *req)
{
    if (!req || req->n < 1)
        return 0;
    long ncells = req->ncells > 0 ? req->ncells : long(req->n) * req->n * req->n;
    return ncells * ElementsPerCell(req->shape);
}

extern "C" int nkb_geom_fill(const nkb_geom_request *req, double *jac, double *df, double *xyz)
{
    if (!req || !jac || !df)
        return SetError(NKB_ERR_INVALID, "nkb_geom_fill: NULL argument");
    if (req->shape != NKB_HEX && req->shape != NKB_PRISM && req->shape != NKB_TET)
        return SetError(NKB_ERR_INVALID, "nkb_geom_fill: bad shape %d", req->shape);
    const int epc     = ElementsPerCell(req->shape);
    const long ncells = req->ncells > 0 ? req->ncells : long(req->n) * req->n * req->n;
    const long nelmt  = ncells * epc;
    const int nq0 = req->nq[0], nq1 = req->nq[1], nq2 = req->nq[2];
    const long nt     = long(nq0) * nq1 * nq2;
    if (!req->deformed && req->amp != 0.0)
        return SetError(NKB_ERR_INVALID, "nkb_geom_fill: curved geometry must be deformed");
    for (int d = 0; d < 3; ++d)
        if (!req->z[d])
            return SetError(NKB_ERR_INVALID, "nkb_geom_fill: missing points for dir %d", d);
    const long ncol = req->deformed ? nelmt * nt : nelmt;

    // cells split over host threads: every element writes its own columns
    auto fill_cells = [&](long c0, long c1) {
    for (long c = c0; c < c1; ++c)
    {
        int cell = req->cells ? req->cells[c] : int(c);
        for (int s = 0; s < epc; ++s)
        {
            long e       = c * epc + s;
            Affine A     = CellMap(req->shape, req->n, cell, s);
            long npts    = req->deformed ? nt : 1;
            for (long q = 0; q < npts; ++q)
            {
                int i = int(q % nq0), j = int((q / nq0) % nq1), k = int(q / (long(nq0) * nq1));
                double eta[3] = {req->z[0][i], req->z[1][j], req->z[2][k]};
                if (!req->deformed)
                    eta[0] = eta[1] = eta[2] = -0.5; // any interior point: affine
                double xp[3], Ji[3][3], jv;
                AtPoint(req->shape, req->amp, A, eta, jv, Ji, xp);
                long col  = req->deformed ? e * nt + q : e;
                jac[col]  = jv;
                for (int kk = 0; kk < 3; ++kk)
                    for (int jj = 0; jj < 3; ++jj)
                        df[(kk * 3 + jj) * ncol + col] = Ji[jj][kk];
                if (xyz && req->deformed)
                    for (int a = 0; a < 3; ++a)
                        xyz[a * nelmt * nt + e * nt + q] = xp[a];
            }
            if (xyz && !req->deformed)
            {
                // coordinates still per point
                for (long q = 0; q < nt; ++q)
                {
                    int i = int(q % nq0), j = int((q / nq0) % nq1), k = int(q / (long(nq0) * nq1));
                    double eta[3] = {req->z[0][i], req->z[1][j], req->z[2][k]}, xi[3], x[3], xp[3],
                           Jc[3][3];
                    Uncollapse(req->shape, eta, xi);
                    for (int a = 0; a < 3; ++a)
                    {
                        x[a] = A.x0[a];
                        for (int b = 0; b < 3; ++b)
                            x[a] += A.M[a][b] * 0.5 * (xi[b] + 1.0);
                    }
                    CurvedMap(req->amp, x, xp, Jc);
                    for (int a = 0; a < 3; ++a)
                        xyz[a * nelmt * nt + e * nt + q] = xp[a];
                }
            }
        }
    }
    };
    const long work     = ncells * epc * (req->deformed ? nt : 1);
    const int nthreads  = int(std::max<long>(1, std::min<long>({long(std::thread::hardware_concurrency()),
                                                              32L, work / 65536 + 1, ncells})));
    if (nthreads == 1)
        fill_cells(0, ncells);
    else
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t)
            pool.emplace_back(fill_cells, ncells * t / nthreads, ncells * (t + 1) / nthreads);
        for (std::thread &th : pool)
            th.join();
    }
    return NKB_OK;
}

// Tensor-product C0 numbering of a hex box with aligned local axes. Per
// direction the 1-D dofs are the n+1 vertices and n*(nm-2) edge-interior
// modes; a 3-D mode is a triple of 1-D dofs. A triple touching x, y or z in
// {0, 1} lies on the boundary: those are the Dirichlet coefficients and are
// numbered first (AssemblyMapCG's Dirichlet-first global ordering,
// AssemblyMapCG.cpp:1512-2045). Shared edges are traversed in the same
// direction by both neighbours, so every sign is +1.
extern "C" int nkb_hex_box_assembly(int n, int nm, int *map, int *nglob, int *ndir)
{
    if (n < 1 || nm < 2 || !map || !nglob || !ndir)
        return SetError(NKB_ERR_INVALID, "nkb_hex_box_assembly: bad arguments");
    const long N1 = long(n) * (nm - 1) + 1;
    const long N3 = N1 * N1 * N1;
    if (N3 > 0x7fffffffL)
        return SetError(NKB_ERR_INVALID, "nkb_hex_box_assembly: too many dofs");
    // 1-D dof id: vertex v -> v*(nm-1); interior mode m of cell c -> c*(nm-1) + (m-1)
    auto dof1 = [&](int c, int p) -> long {
        if (p == 0)
            return long(c) * (nm - 1);
        if (p == 1)
            return long(c + 1) * (nm - 1);
        return long(c) * (nm - 1) + (p - 1);
    };
    // Boundary dofs first, then interior ones, each set in lexicographic
    // (c, b, a) order; both ranks have closed forms: a boundary plane (c = 0
    // or N1-1) holds N1^2 boundary dofs, an interior plane 4 N1 - 4 (its first
    // and last rows whole, two of every other row).
    const long M1 = N1 - 2, ndirc = N3 - M1 * M1 * M1;
    auto onb = [&](long x) { return x == 0 || x == N1 - 1; };
    auto rank = [&](long a, long b, long c) -> long {
        if (!(onb(a) || onb(b) || onb(c)))
            return ndirc + ((c - 1) * M1 + (b - 1)) * M1 + (a - 1);
        const long before = c == 0 ? 0 : N1 * N1 + (c - 1) * (4 * N1 - 4);
        if (onb(c))
            return before + b * N1 + a;
        const long row = b == 0 ? 0 : N1 + (b - 1) * 2;
        if (onb(b))
            return before + row + a;
        return before + row + (a == 0 ? 0 : 1);
    };
    const long nelmt = long(n) * n * n, nc = long(nm) * nm * nm;
    const int nthreads = int(std::max<long>(
        1, std::min<long>({long(std::thread::hardware_concurrency()), 32L, nelmt * nc / 262144 + 1})));
    auto fill = [&](long e0, long e1) {
        for (long e = e0; e < e1; ++e)
        {
            int cx = int(e % n), cy = int((e / n) % n), cz = int(e / (long(n) * n));
            for (int r = 0; r < nm; ++r)
                for (int q = 0; q < nm; ++q)
                    for (int p = 0; p < nm; ++p)
                        map[e * nc + (long(r) * nm + q) * nm + p] =
                            int(rank(dof1(cx, p), dof1(cy, q), dof1(cz, r)));
        }
    };
    if (nthreads == 1)
        fill(0, nelmt);
    else
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t)
            pool.emplace_back(fill, nelmt * t / nthreads, nelmt * (t + 1) / nthreads);
        for (std::thread &th : pool)
            th.join();
    }
    *nglob = int(N3);
    *ndir  = int(ndirc);
    return NKB_OK;
}
