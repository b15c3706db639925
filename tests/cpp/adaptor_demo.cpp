// Drives the C++ Collections mirror (nektar_b200/adaptor/nkb_collections.hpp)
// the way a Nektar++ Collection would: factory lookup by OperatorKey with the
// eB200 implementation type, Helmholtz apply with UpdateFactors, an
// IProductWRTDerivBase apply with three input fields, a LinearADR apply with
// UpdateVarcoeffs, then the
// GlobalLinSysIterativeFull solve. Prints one JSON line. Exit codes: 0 ok,
// 3 NekError raised (e.g. no CUDA device), 1 other failure.
#include "../../nektar_b200/adaptor/nkb_collections.hpp"

#include <cmath>
#include <cstdio>

using namespace nkb::collections;

int main()
{
    const int n = 3, nm = 5, nq = 6;
    CollectionData d;
    d.shape    = eHexahedron;
    d.nm       = nm;
    d.nq       = {nq, nq, nq};
    d.ptype    = {NKB_GLL, NKB_GLL, NKB_GLL};
    d.deformed = true;
    for (int k = 0; k < 3; ++k)
    {
        d.z[k].resize(nq);
        d.w[k].resize(nq);
        d.D[k].resize(nq * nq);
        d.bdata[k].resize(nm * nq);
        Check(nkb_points(NKB_GLL, nq, d.z[k].data(), d.w[k].data(), d.D[k].data()));
        if (nkb_basis(NKB_MODIFIED_A, nm, nq, d.z[k].data(), d.D[k].data(), d.bdata[k].data(),
                      nullptr) < 0)
            return 1;
    }
    nkb_geom_request req{};
    req.shape    = NKB_HEX;
    req.n        = n;
    req.amp      = 0.05;
    req.nq[0] = req.nq[1] = req.nq[2] = nq;
    for (int k = 0; k < 3; ++k)
        req.z[k] = d.z[k].data();
    req.deformed = 1;
    d.nelmt      = int(nkb_geom_nelmt(&req));
    const long nt = long(nq) * nq * nq, nc = long(nm) * nm * nm;
    d.jac.resize(d.nelmt * nt);
    d.df.resize(9 * d.nelmt * nt);
    Check(nkb_geom_fill(&req, d.jac.data(), d.df.data(), nullptr));
    std::vector<int> map(d.nelmt * nc);
    int nglob = 0, ndir = 0;
    Check(nkb_hex_box_assembly(n, nm, map.data(), &nglob, &ndir));

    // a collection of per-direction orders is refused before any device work
    int aniso = 0;
    try
    {
        RegisterB200Operators();
        CollectionData da = d;
        da.nmodes         = {nm, nm + 1, nm};
        FactorMap fa;
        GetOperatorFactory().CreateInstance(OperatorKey(eHexahedron, eHelmholtz, eB200, false),
                                            da, fa);
    }
    catch (const NekError &e)
    {
        aniso = e.Code();
    }
    try
    {
        FactorMap f;
        f.lambda = 1.5;
        auto op  = GetOperatorFactory().CreateInstance(OperatorKey(eHexahedron, eHelmholtz, eB200,
                                                                   false),
                                                       d, f);
        Array1D x(op->GetInputSize()), y(op->GetOutputSize()), e1, e2, wsp;
        for (size_t i = 0; i < x.size(); ++i)
            x[i] = std::sin(0.37 * double(i));
        (*op)(x, y, e1, e2, wsp);
        double ny = 0.0;
        for (double v : y)
            ny += v * v;
        bool threw = false;
        try
        {
            (*op)(0, x, y, wsp);
        }
        catch (const NekError &)
        {
            threw = true; // "Not valid for this operator." as Helmholtz.cpp:604-610
        }
        // IProductWRTDerivBase: three field components in, coefficients out
        auto ipd = GetOperatorFactory().CreateInstance(
            OperatorKey(eHexahedron, eIProductWRTDerivBase, eB200, false), d, f);
        Array1D f0(ipd->GetInputSize()), f1(f0.size()), f2(f0.size()), g(ipd->GetOutputSize());
        for (size_t i = 0; i < f0.size(); ++i)
        {
            f0[i] = std::cos(0.11 * double(i));
            f1[i] = std::cos(0.11 * double(i) + 1.0);
            f2[i] = std::cos(0.11 * double(i) + 2.0);
        }
        (*ipd)(f0, f1, f2, g, wsp);
        double ng = 0.0;
        for (double v : g)
            ng += v * v;
        // LinearAdvectionDiffusionReaction with a velocity field
        auto adr = GetOperatorFactory().CreateInstance(
            OperatorKey(eHexahedron, eLinearAdvectionDiffusionReaction, eB200, false), d, f);
        VarCoeffMap vc;
        vc.velx.resize(f0.size());
        vc.vely.resize(f0.size());
        vc.velz.resize(f0.size());
        for (size_t i = 0; i < f0.size(); ++i)
        {
            vc.velx[i] = 1.0 + 0.1 * std::sin(0.05 * double(i));
            vc.vely[i] = -0.5;
            vc.velz[i] = 0.25 * std::cos(0.02 * double(i));
        }
        adr->UpdateVarcoeffs(vc);
        Array1D ya(adr->GetOutputSize());
        (*adr)(x, ya, e1, e2, wsp);
        double na = 0.0;
        for (double v : ya)
            na += v * v;
        auto helm = std::dynamic_pointer_cast<Helmholtz_B200>(op);
        GlobalLinSysIterativeFullB200 sys({helm}, map, nglob, ndir);
        Array1D b(x), sol(x.size(), 0.0);
        nkb_cg_report r = sys.Solve(b, sol, 1e-10);
        std::printf("{\"helmholtz_norm2\": %.17g, \"iproduct_deriv_norm2\": %.17g, "
                    "\"linear_adr_norm2\": %.17g, "
                    "\"dir_call_threw\": %d, \"cg_iterations\": %d, "
                    "\"cg_rel_residual\": %.6g, \"nelmt\": %d, \"per_direction_orders\": %d}\n",
                    ny, ng, na, int(threw), r.iterations, r.rel_residual, d.nelmt, aniso);
        return 0;
    }
    catch (const NekError &e)
    {
        std::printf("{\"nekerror\": %d, \"what\": \"%s\", \"per_direction_orders\": %d}\n",
                    e.Code(), e.what(), aniso);
        return 3;
    }
}
