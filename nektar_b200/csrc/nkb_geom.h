// Geometry of the structured test meshes (unit-cube boxes of n^3 cells,
// hexahedra or cells split into 2 prisms / 6 tetrahedra, optionally curved
// by x' = x + amp sin(pi x) sin(pi y) sin(pi z)): the analytic Jacobian and
// its inverse at one quadrature point. Shared by the host fill
// (nkb_geom_fill) and the device fill (nkb_geom_fill_device).
#pragma once

#include "../../include/nektar_b200.h"

#include <cmath>

#ifdef __CUDACC__
#define NKB_HD __host__ __device__
#else
#define NKB_HD
#endif

namespace nkb
{
namespace geom
{
struct Affine
{
    double x0[3];
    double M[3][3]; // x = x0 + M (xi + 1)/2, M[k][i] = d x_k / d ((xi_i+1)/2)
};

NKB_HD inline int ElementsPerCell(int shape)
{
    return shape == NKB_HEX ? 1 : (shape == NKB_PRISM ? 2 : 6);
}

NKB_HD inline double Det3(const double A[3][3])
{
    return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
           A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

// Affine map of sub-element s of cell (cx, cy, cz), h = 1/n.
NKB_HD inline Affine CellMap(int shape, int n, int cell, int s)
{
    const double h = 1.0 / n;
    int cx = cell % n, cy = (cell / n) % n, cz = cell / (n * n);
    double o[3] = {cx * h, cy * h, cz * h};
    Affine A;
    for (int k = 0; k < 3; ++k)
    {
        A.x0[k] = 0.0;
        for (int l = 0; l < 3; ++l)
            A.M[k][l] = 0.0;
    }
    if (shape == NKB_HEX)
    {
        for (int k = 0; k < 3; ++k)
        {
            A.x0[k]    = o[k];
            A.M[k][k]  = h;
        }
    }
    else if (shape == NKB_PRISM)
    {
        // standard prism: triangle {xi0 + xi2 <= 0} in (xi0, xi2), extruded in xi1
        if (s == 0)
        {
            for (int k = 0; k < 3; ++k)
            {
                A.x0[k]   = o[k];
                A.M[k][k] = h;
            }
        }
        else
        {
            // the other half x_l + z_l >= 1: x_l = 1 - a, z_l = 1 - c
            A.x0[0]   = o[0] + h;
            A.x0[1]   = o[1];
            A.x0[2]   = o[2] + h;
            A.M[0][0] = -h;
            A.M[1][1] = h;
            A.M[2][2] = -h;
        }
    }
    else
    {
        // Kuhn split: tet s visits 0 -> e_a -> e_a + e_b -> (1,1,1)
        static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2},
                                       {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
        double v[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {1, 1, 1}};
        v[1][perm[s][0]] = 1;
        v[2][perm[s][0]] = 1;
        v[2][perm[s][1]] = 1;
        double M[3][3];
        for (int k = 0; k < 3; ++k)
            for (int i = 0; i < 3; ++i)
                M[k][i] = h * (v[i + 1][k] - v[0][k]);
        if (Det3(M) < 0)
            for (int k = 0; k < 3; ++k)
            {
                const double t = M[k][0];
                M[k][0]        = M[k][1];
                M[k][1]        = t;
            }
        for (int k = 0; k < 3; ++k)
        {
            A.x0[k] = o[k];
            for (int i = 0; i < 3; ++i)
                A.M[k][i] = M[k][i];
        }
    }
    return A;
}

// standard coordinates xi of a quadrature point given in the collapsed
// coordinates eta of the shape (Nektar's collapsed systems).
NKB_HD inline void Uncollapse(int shape, const double eta[3], double xi[3])
{
    if (shape == NKB_HEX)
    {
        xi[0] = eta[0];
        xi[1] = eta[1];
        xi[2] = eta[2];
    }
    else if (shape == NKB_PRISM)
    {
        xi[2] = eta[2];
        xi[1] = eta[1];
        xi[0] = 0.5 * (1.0 + eta[0]) * (1.0 - eta[2]) - 1.0;
    }
    else
    {
        xi[2] = eta[2];
        xi[1] = 0.5 * (1.0 + eta[1]) * (1.0 - eta[2]) - 1.0;
        xi[0] = 0.5 * (1.0 + eta[0]) * (-xi[1] - xi[2]) - 1.0;
    }
}

// x' = x + amp S(x) (every coordinate), S = sin(pi x) sin(pi y) sin(pi z)
NKB_HD inline void CurvedMap(double amp, const double x[3], double xp[3], double Jm[3][3])
{
    const double sx = sin(M_PI * x[0]), sy = sin(M_PI * x[1]),
                 sz = sin(M_PI * x[2]);
    const double cx = cos(M_PI * x[0]), cy = cos(M_PI * x[1]),
                 cz = cos(M_PI * x[2]);
    const double S     = sx * sy * sz;
    const double dS[3] = {M_PI * cx * sy * sz, M_PI * sx * cy * sz, M_PI * sx * sy * cz};
    for (int k = 0; k < 3; ++k)
    {
        xp[k] = x[k] + amp * S;
        for (int l = 0; l < 3; ++l)
            Jm[k][l] = (k == l ? 1.0 : 0.0) + amp * dS[l];
    }
}


// jac = |det J|, Ji[i][k] = d xi_i / d x_k and the mapped point xp at the
// collapsed coordinates eta of sub-element s of a cell (the fill's order of
// operations)
NKB_HD inline void AtPoint(int shape, double amp, const Affine &A, const double eta[3], double &jac,
                           double Ji[3][3], double xp[3])
{
    double xi[3], x[3], Jc[3][3], J[3][3];
    Uncollapse(shape, eta, xi);
    for (int a = 0; a < 3; ++a)
    {
        x[a] = A.x0[a];
        for (int b = 0; b < 3; ++b)
            x[a] += A.M[a][b] * 0.5 * (xi[b] + 1.0);
    }
    CurvedMap(amp, x, xp, Jc);
    // J[k][i] = d x'_k / d xi_i = sum_l Jc[k][l] M[l][i] / 2
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
        {
            double v = 0.0;
            for (int l = 0; l < 3; ++l)
                v += Jc[a][l] * A.M[l][b];
            J[a][b] = 0.5 * v;
        }
    double det = Det3(J);
    Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
    Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
    Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
    Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    jac      = fabs(det);
}
} // namespace geom
} // namespace nkb
