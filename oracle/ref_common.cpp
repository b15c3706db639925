// Test infrastructure only: part of the oracle, never of the product.
//
// Shape-independent half of the reference harness (see ref_harness.cpp):
//  * thin C wrappers around the reference's own Polylib routines (compiled in
//    place from LibUtilities/Polylib/Polylib.cpp), used to pin the product's
//    quadrature and basis tables;
//  * a restatement of Basis::GenBasis for Modified_A/B/C (Basis.cpp:466-644)
//    on top of the reference Polylib::jacobfd, with dbdata = D * bdata as the
//    reference's Blas::Dgemm call computes it;
//  * the per-direction points/weights/derivative tables of GaussPoints
//    (GaussPoints.cpp:79-140 and 193-240) and the Radau weight factors of
//    Operator.hpp:592-625 (SetUpZW);
//  * the CPU preconditioned-CG driver used as the timed CPU baseline of the
//    global solve: NekLinSysIterCG::DoConjugateGradient
//    (NekLinSysIterCG.cpp:118-372) with the AssemblyMapCG gather/assemble
//    (AssemblyMapCG.cpp:2804-2886) and the diagonal preconditioner apply
//    (PreconditionerDiagonal.cpp:159-189), with the element operator supplied
//    as a callback (the reference kernels of ref_harness.cpp).

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

#include <pthread.h>
#include <sched.h>

#include <LibUtilities/Polylib/Polylib.h>

extern "C" void nkref_pin_thread(int t);

namespace
{
// host CPUs the worker threads are pinned to (worker t -> cpus[t % n]);
// empty: no pinning
std::vector<int> g_cpus;

// Points types, numbered as LibUtilities::PointsType (PointsType.h:43-)
enum
{
    kGaussLobattoLegendre  = 4,
    kGaussRadauMAlpha1Beta0 = 11,
    kGaussRadauMAlpha2Beta0 = 12
};

template <class F> void ParallelFor(long n, int nthreads, F &&f)
{
    nthreads = std::max(1, nthreads);
    if (nthreads == 1 || n < 4096)
    {
        f(0L, n, 0);
        return;
    }
    std::vector<std::thread> ts;
    long chunk = (n + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; ++t)
    {
        long a = t * chunk, b = std::min(n, a + chunk);
        if (a >= b)
        {
            break;
        }
        ts.emplace_back([&f, a, b, t] {
            nkref_pin_thread(t);
            f(a, b, t);
        });
    }
    for (auto &t : ts)
    {
        t.join();
    }
}

} // namespace

extern "C"
{

    // ---- worker-thread pinning (timed CPU baseline) ------------------------
    void nkref_set_cpus(int n, const int *cpus)
    {
        g_cpus.assign(cpus, cpus + std::max(0, n));
    }
    void nkref_pin_thread(int t)
    {
        if (g_cpus.empty())
            return;
        cpu_set_t set;
        CPU_ZERO(&set);
        CPU_SET(g_cpus[size_t(t) % g_cpus.size()], &set);
        pthread_setaffinity_np(pthread_self(), sizeof(set), &set);
    }

    // ---- Polylib (reference code) -------------------------------------------
    void nkref_zwglj(double *z, double *w, int np, double alpha, double beta)
    {
        Polylib::zwglj(z, w, np, alpha, beta);
    }
    void nkref_zwgrjm(double *z, double *w, int np, double alpha, double beta)
    {
        Polylib::zwgrjm(z, w, np, alpha, beta);
    }
    void nkref_Dglj(double *D, const double *z, int np, double alpha, double beta)
    {
        Polylib::Dglj(D, z, np, alpha, beta);
    }
    void nkref_Dgrjm(double *D, const double *z, int np, double alpha, double beta)
    {
        Polylib::Dgrjm(D, z, np, alpha, beta);
    }
    void nkref_jacobfd(int np, const double *z, double *poly, double *polyd, int n, double alpha,
                       double beta)
    {
        Polylib::jacobfd(np, z, poly, polyd, n, alpha, beta);
    }

    // Points of type ptype: z, w (raw Nektar weights) and the derivative matrix
    // as Points::GetD()->GetPtr() stores it, D[k*np + i] = d l_k / dz (z_i).
    // Polylib's Dglj / Dgrjm fill D[i*np + j] = pd[j] / (pd[i] (z_j - z_i)),
    // which is d l_i / dz (z_j) (Polylib.cpp:833-912): already that layout,
    // and GaussPoints.cpp:279-280 copies it unchanged.
    int nkref_points(int ptype, int np, double *z, double *w, double *D)
    {
        std::vector<double> Dp(std::size_t(np) * np);
        using namespace Polylib;
        switch (ptype)
        {
            case kGaussLobattoLegendre:
                zwglj(z, w, np, 0.0, 0.0);
                Dglj(Dp.data(), z, np, 0.0, 0.0);
                break;
            case kGaussRadauMAlpha1Beta0:
                zwgrjm(z, w, np, 1.0, 0.0);
                Dgrjm(Dp.data(), z, np, 1.0, 0.0);
                break;
            case kGaussRadauMAlpha2Beta0:
                zwgrjm(z, w, np, 2.0, 0.0);
                Dgrjm(Dp.data(), z, np, 2.0, 0.0);
                break;
            default:
                return -1;
        }
        std::copy(Dp.begin(), Dp.end(), D);
        return 0;
    }

    // Operator.hpp:592-625: weight factor applied by SetUpZW
    double nkref_weight_factor(int ptype)
    {
        if (ptype == kGaussRadauMAlpha1Beta0)
        {
            return 0.5;
        }
        if (ptype == kGaussRadauMAlpha2Beta0)
        {
            return 0.25;
        }
        return 1.0;
    }

    // Basis::GenBasis restated for Modified_A (btype 4), Modified_B (5),
    // Modified_C (6); numbering as LibUtilities::BasisType. D as returned by
    // nkref_points (column-major). Output sizes: nb * np with nb the number of
    // tabulated modes for the basis type.
    int nkref_basis(int btype, int nm, int np, const double *z, const double *D, double *bdata,
                    double *dbdata)
    {
        using Polylib::jacobfd;
        std::size_t nb = 0;
        if (btype == 4)
        {
            // Basis.cpp:466-497
            for (int i = 0; i < np; ++i)
            {
                bdata[i]      = 0.5 * (1 - z[i]);
                bdata[np + i] = 0.5 * (1 + z[i]);
            }
            double *mode = bdata + 2 * np;
            for (int p = 2; p < nm; ++p, mode += np)
            {
                jacobfd(np, z, mode, nullptr, p - 2, 1.0, 1.0);
                for (int i = 0; i < np; ++i)
                {
                    mode[i] *= bdata[i] * bdata[np + i];
                }
            }
            nb = nm;
        }
        else if (btype == 5 || btype == 6)
        {
            // Modified_B, Basis.cpp:499-588
            std::vector<double> B(std::size_t(nm) * (nm + 1) / 2 * np);
            for (int i = 0; i < np; ++i)
            {
                B[i]      = 0.5 * (1 - z[i]);
                B[np + i] = 0.5 * (1 + z[i]);
            }
            double *mode = B.data() + 2 * np;
            for (int q = 2; q < nm; ++q, mode += np)
            {
                jacobfd(np, z, mode, nullptr, q - 2, 1.0, 1.0);
                for (int i = 0; i < np; ++i)
                {
                    mode[i] *= B[i] * B[np + i];
                }
            }
            for (int i = 0; i < np; ++i)
            {
                mode[i] = 0.5 * (1 - z[i]);
            }
            mode += np;
            for (int q = 2; q < nm; ++q, mode += np)
            {
                jacobfd(np, z, mode, nullptr, q - 2, 1.0, 1.0);
                for (int i = 0; i < np; ++i)
                {
                    mode[i] *= B[i] * B[np + i];
                }
            }
            const double *one_m_z_pow = B.data();
            const double *one_p_z     = B.data() + np;
            for (int p = 2; p < nm; ++p)
            {
                for (int i = 0; i < np; ++i)
                {
                    mode[i] = B[i] * one_m_z_pow[i];
                }
                one_m_z_pow = mode;
                mode += np;
                for (int q = 1; q < nm - p; ++q, mode += np)
                {
                    jacobfd(np, z, mode, nullptr, q - 1, 2 * p - 1, 1.0);
                    for (int i = 0; i < np; ++i)
                    {
                        mode[i] *= one_m_z_pow[i] * one_p_z[i];
                    }
                }
            }
            if (btype == 5)
            {
                nb = std::size_t(nm) * (nm + 1) / 2;
                std::copy(B.begin(), B.end(), bdata);
            }
            else
            {
                // Modified_C: phi^c_{pqr} = phi^b_{p+q, r} (Basis.cpp:590-644)
                std::size_t boff = 0, off = 0;
                for (int p = 0; p < nm; ++p)
                {
                    std::size_t N = std::size_t(np) * (nm - p) * (nm - p + 1) / 2;
                    std::copy(B.begin() + boff, B.begin() + boff + N, bdata + off);
                    boff += std::size_t(np) * (nm - p);
                    off += N;
                }
                nb = std::size_t(nm) * (nm + 1) * (nm + 2) / 6;
            }
        }
        else
        {
            return -1;
        }
        // dbdata = D * bdata  (column-major np x np times np x nb)
        for (std::size_t m = 0; m < nb; ++m)
        {
            for (int i = 0; i < np; ++i)
            {
                double s = 0.0;
                for (int k = 0; k < np; ++k)
                {
                    s += D[std::size_t(k) * np + i] * bdata[m * np + k];
                }
                dbdata[m * np + i] = s;
            }
        }
        return int(nb);
    }

    // ---- global PCG driver for the CPU baseline -----------------------------
    typedef void (*nkref_apply_fn)(void *op, const double *in, double *out0, double *out1,
                                   double *out2);

    // Solve A x = b on the non-Dirichlet part of the global system, with
    // A = Assemble o (element Helmholtz) o GlobalToLocal. b_glob is the
    // assembled right-hand side (all nGlob entries, Dirichlet first),
    // x_glob on output holds the solution in [nDir, nGlob) and 0 on the
    // Dirichlet part, exactly as NekLinSysIterCG returns it. The assemble is
    // written as a gather over a global->local CSR (asm_ptr, asm_idx) so that
    // threads never write the same global entry. Returns iterations done.
    int nkref_pcg_solve(int nGlob, int nDir, long nLoc, const int *map, const double *sign,
                        const int *asm_ptr, const long *asm_idx, nkref_apply_fn apply, void *op,
                        const double *diag_inv, const double *b_glob, double *x_glob, double tol,
                        int maxit, int nthreads, int max_iters_to_run, double *err_out)
    {
        const int nNonDir = nGlob - nDir;
        std::vector<double> w(nGlob, 0.0), s(nGlob, 0.0), p(nNonDir, 0.0), r(nNonDir, 0.0),
            q(nNonDir, 0.0);
        std::vector<double> wl(nLoc), sl(nLoc);

        auto dot = [&](const double *a, const double *b, long n) {
            std::vector<double> part(std::max(1, nthreads), 0.0);
            ParallelFor(n, nthreads, [&](long i0, long i1, int t) {
                double acc = 0.0;
                for (long i = i0; i < i1; ++i)
                {
                    acc += a[i] * b[i];
                }
                part[t] = acc;
            });
            double acc = 0.0;
            for (double v : part)
            {
                acc += v;
            }
            return acc;
        };
        auto matvec = [&]() {
            // GlobalToLocal (AssemblyMapCG.cpp:2804-2827)
            ParallelFor(nLoc, nthreads, [&](long i0, long i1, int) {
                for (long i = i0; i < i1; ++i)
                {
                    wl[i] = sign ? sign[i] * w[map[i]] : w[map[i]];
                }
            });
            apply(op, wl.data(), sl.data(), nullptr, nullptr);
            // Assemble (AssemblyMapCG.cpp:2860-2886)
            ParallelFor(nGlob, nthreads, [&](long g0, long g1, int) {
                for (long g = g0; g < g1; ++g)
                {
                    double acc = 0.0;
                    for (int k = asm_ptr[g]; k < asm_ptr[g + 1]; ++k)
                    {
                        long l = asm_idx[k];
                        acc += sign ? sign[l] * sl[l] : sl[l];
                    }
                    s[g] = acc;
                }
            });
        };
        auto precon = [&]() {
            ParallelFor(nNonDir, nthreads, [&](long i0, long i1, int) {
                for (long i = i0; i < i1; ++i)
                {
                    w[nDir + i] = r[i] * diag_inv[i];
                }
            });
        };

        std::copy(b_glob + nDir, b_glob + nGlob, r.begin());
        std::fill(x_glob, x_glob + nGlob, 0.0);
        double eps     = dot(r.data(), r.data(), nNonDir);
        double rhs_mag = dot(b_glob, b_glob, nGlob);
        rhs_mag        = (rhs_mag > 1.0e-6) ? rhs_mag : 1.0;
        tol            = std::fmax(tol, 1.0e-16);
        int iters      = 0;
        if (eps < tol * tol * rhs_mag)
        {
            if (err_out)
            {
                *err_out = std::sqrt(eps / rhs_mag);
            }
            return 0;
        }
        precon();
        matvec();
        double rho   = dot(r.data(), w.data() + nDir, nNonDir);
        double mu    = dot(s.data() + nDir, w.data() + nDir, nNonDir);
        double beta  = 0.0;
        double alpha = rho / mu;
        iters        = 1;
        while (true)
        {
            if (iters > maxit || (max_iters_to_run > 0 && iters > max_iters_to_run))
            {
                break;
            }
            ParallelFor(nNonDir, nthreads, [&](long i0, long i1, int) {
                for (long i = i0; i < i1; ++i)
                {
                    p[i] = beta * p[i] + w[nDir + i];
                    q[i] = beta * q[i] + s[nDir + i];
                    x_glob[nDir + i] += alpha * p[i];
                    r[i] -= alpha * q[i];
                }
            });
            precon();
            matvec();
            double rho_new = dot(r.data(), w.data() + nDir, nNonDir);
            mu             = dot(s.data() + nDir, w.data() + nDir, nNonDir);
            eps            = dot(r.data(), r.data(), nNonDir);
            iters++;
            if (eps < tol * tol * rhs_mag)
            {
                break;
            }
            beta  = rho_new / rho;
            alpha = rho_new / (mu - rho_new * beta / alpha);
            rho   = rho_new;
        }
        if (err_out)
        {
            *err_out = std::sqrt(eps / rhs_mag);
        }
        return iters;
    }
}
