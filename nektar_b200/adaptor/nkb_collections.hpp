// C++ host side of the B200 path, mirroring the reference's Collections
// plugin interface (Collections/Operator.h:43-245) on top of the C ABI of
// include/nektar_b200.h:
//
//   * Operator: abstract operator with operator()(in, out0, out1, out2, wsp),
//     operator()(dir, in, out, wsp), UpdateFactors, GetInputSize/GetOutputSize;
//   * OperatorKey (shape, operator type, implementation type, nodal) and a
//     factory keyed by it (GetOperatorFactory().CreateInstance), with the new
//     implementation type eB200 registered for Hex/Prism/Tet x BwdTrans,
//     IProductWRTBase, IProductWRTDerivBase, PhysDeriv, Helmholtz,
//     LinearAdvectionDiffusionReaction;
//   * GlobalLinSysIterativeFullB200: the GlobalLinSysIterativeFull solve.
//
// Errors: a failing status from the C ABI throws NekError with the
// library's message, as NEKERROR / ASSERTL0 do in the reference
// (LibUtilities/BasicUtils/ErrorUtil.hpp:57,210-235). Arrays are plain host
// vectors here; in a Nektar++ build the same classes take Array<OneD, ...>
// (LibUtilities/BasicUtils/SharedArray.hpp) and hand their data pointers to
// the C ABI the same way.
#pragma once

#include "../../include/nektar_b200.h"

#include <array>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace nkb
{
namespace collections
{

class NekError : public std::runtime_error
{
public:
    NekError(int code, const std::string &msg) : std::runtime_error(msg), m_code(code)
    {
    }
    int Code() const
    {
        return m_code;
    }

private:
    int m_code;
};

inline void Check(int rc)
{
    if (rc != NKB_OK)
        throw NekError(rc, std::string("nektar_b200: ") + nkb_last_error());
}

// numbering of Collections::OperatorType / ImplementationType (Operator.h:62-93)
enum OperatorType
{
    eBwdTrans                         = NKB_BWDTRANS,
    eHelmholtz                        = NKB_HELMHOLTZ,
    eLinearAdvectionDiffusionReaction = NKB_LINEAR_ADR,
    eIProductWRTBase      = NKB_IPRODUCT,
    eIProductWRTDerivBase = NKB_IPRODUCT_DERIV,
    ePhysDeriv            = NKB_PHYSDERIV
};
enum ImplementationType
{
    eNoImpType,
    eNoCollection,
    eIterPerExp,
    eStdMat,
    eSumFac,
    eMatrixFree,
    eB200, // the new implementation type, appended before SIZE_ImplementationType
    SIZE_ImplementationType
};
enum ShapeType
{
    eTetrahedron = NKB_TET,
    ePrism       = NKB_PRISM,
    eHexahedron  = NKB_HEX
};

using Array1D = std::vector<double>;
// StdRegions::FactorMap subset the Helmholtz operator reads (Helmholtz.cpp:615-691)
struct FactorMap
{
    double lambda = 1.0;
    std::array<double, 6> coeffD = {1, 0, 1, 0, 0, 1}; // D00 D01 D11 D02 D12 D22
    double tau                  = 0.0;                 // eFactorTau != 0: variable diffusion
};

// StdRegions::VarCoeffMap subset LinearADR reads: eVarCoeffVelX/Y/Z, one
// value per quadrature point of the collection
struct VarCoeffMap
{
    Array1D velx, vely, velz;
};

// what a Collection hands its operator: basis tables, points, geometry
// (LocalRegions expansions + CoalescedGeomData in the reference)
struct CollectionData
{
    ShapeType shape;
    int nm;
    // modes per direction as the expansions report them (GetBasisNumModes(0..2));
    // zeros mean nm in every direction
    std::array<int, 3> nmodes{};
    std::array<int, 3> nq, ptype;
    int nelmt;
    bool deformed;
    std::array<Array1D, 3> bdata, w, z, D;
    Array1D jac, df;
    int device = 0;
};

class Operator
{
public:
    virtual ~Operator() = default;
    virtual void operator()(const Array1D &input, Array1D &output0, Array1D &output1,
                            Array1D &output2, Array1D &wsp) = 0;
    virtual void operator()(int dir, const Array1D &input, Array1D &output, Array1D &wsp) = 0;
    virtual void UpdateFactors(const FactorMap &)
    {
        throw NekError(NKB_ERR_INVALID, "This method needs to be re-implemented in derived "
                                        "operator class.");
    }
    virtual void UpdateVarcoeffs(VarCoeffMap &)
    {
        throw NekError(NKB_ERR_INVALID, "This method needs to be re-implemented in derived "
                                        "operator class. Make sure it is implemented for the "
                                        "operator in the .opt file");
    }
    unsigned GetInputSize() const
    {
        return m_in;
    }
    unsigned GetOutputSize() const
    {
        return m_out;
    }
    unsigned GetNumElmt() const
    {
        return m_nelmt;
    }
    unsigned GetWspSize() const
    {
        return 0;
    }

protected:
    unsigned m_in = 0, m_out = 0, m_nelmt = 0;
};
using OperatorSharedPtr = std::shared_ptr<Operator>;
using OperatorKey       = std::tuple<ShapeType, OperatorType, ImplementationType, bool>;

class OperatorFactory
{
public:
    using Creator = std::function<OperatorSharedPtr(const CollectionData &, const FactorMap &)>;
    OperatorKey RegisterCreatorFunction(const OperatorKey &key, Creator c, const std::string &)
    {
        m_map[key] = std::move(c);
        return key;
    }
    bool ModuleExists(const OperatorKey &key) const
    {
        return m_map.count(key) != 0;
    }
    OperatorSharedPtr CreateInstance(const OperatorKey &key, const CollectionData &d,
                                     const FactorMap &f) const
    {
        auto it = m_map.find(key);
        if (it == m_map.end())
            throw NekError(NKB_ERR_INVALID, "No such operator key in the factory");
        return it->second(d, f);
    }

private:
    std::map<OperatorKey, Creator> m_map;
};

inline OperatorFactory &GetOperatorFactory()
{
    static OperatorFactory f;
    return f;
}

// One C-ABI operator owned by a Collections operator.
class B200OpHandle
{
public:
    B200OpHandle(const CollectionData &d, int optype)
    {
        // the descriptor carries one order for all directions; a collection of
        // per-direction orders (which the reference's MatrixFree operators take
        // through their run-time-sized path) stays with the reference's own
        // implementation
        for (int i = 0; i < 3; ++i)
            if (d.nmodes[i] != 0 && d.nmodes[i] != d.nm)
                throw NekError(NKB_ERR_UNSUPPORTED,
                               "eB200 operators take one order in all directions (modes " +
                                   std::to_string(d.nmodes[0]) + "," +
                                   std::to_string(d.nmodes[1]) + "," +
                                   std::to_string(d.nmodes[2]) + ")");
        nkb_op_desc desc{};
        desc.shape    = d.shape;
        desc.optype   = optype;
        desc.nm       = d.nm;
        desc.nelmt    = d.nelmt;
        desc.deformed = d.deformed ? 1 : 0;
        for (int i = 0; i < 3; ++i)
        {
            desc.nq[i]    = d.nq[i];
            desc.ptype[i] = d.ptype[i];
            desc.bdata[i] = d.bdata[i].empty() ? nullptr : d.bdata[i].data();
            desc.w[i]     = d.w[i].empty() ? nullptr : d.w[i].data();
            desc.z[i]     = d.z[i].empty() ? nullptr : d.z[i].data();
            desc.D[i]     = d.D[i].empty() ? nullptr : d.D[i].data();
        }
        desc.jac       = d.jac.empty() ? nullptr : d.jac.data();
        desc.df        = d.df.empty() ? nullptr : d.df.data();
        desc.precision = NKB_FP64;
        desc.device    = d.device;
        Check(nkb_op_create(&desc, &m_op));
        long in = 0, out = 0;
        Check(nkb_op_sizes(m_op, &in, &out));
        m_in  = unsigned(in);
        m_out = unsigned(out);
    }
    ~B200OpHandle()
    {
        nkb_op_destroy(m_op);
    }
    B200OpHandle(const B200OpHandle &)            = delete;
    B200OpHandle &operator=(const B200OpHandle &) = delete;
    nkb_op *get() const
    {
        return m_op;
    }
    unsigned m_in = 0, m_out = 0;

private:
    nkb_op *m_op = nullptr;
};

// BwdTrans / IProductWRTBase / Helmholtz: single output (Operator.h:148-152)
template <int OPTYPE> class SingleOutput_B200 : public Operator
{
public:
    SingleOutput_B200(const CollectionData &d, const FactorMap &f) : m_h(d, OPTYPE)
    {
        m_in    = m_h.m_in;
        m_out   = m_h.m_out;
        m_nelmt = unsigned(d.nelmt);
        if (OPTYPE == eHelmholtz)
            UpdateFactors(f);
    }
    void operator()(const Array1D &input, Array1D &output0, Array1D &, Array1D &,
                    Array1D &) override
    {
        if (input.size() < m_in || output0.size() < m_out)
            throw NekError(NKB_ERR_INVALID, "array smaller than the operator's size");
        Check(nkb_op_apply(m_h.get(), input.data(), output0.data(), nullptr, nullptr,
                           NKB_HOST_PTRS, nullptr));
    }
    void operator()(int, const Array1D &, Array1D &, Array1D &) override
    {
        throw NekError(NKB_ERR_INVALID, "Not valid for this operator.");
    }
    // Helmholtz_MatrixFree::UpdateFactors (Helmholtz.cpp:615-691)
    void UpdateFactors(const FactorMap &f) override
    {
        if (OPTYPE != eHelmholtz)
            return Operator::UpdateFactors(f);
        static const double id[6] = {1, 0, 1, 0, 0, 1};
        bool isConst              = false;
        for (int c = 0; c < 6; ++c)
            isConst = isConst || f.coeffD[c] != id[c];
        int mode = f.tau != 0.0 ? NKB_DIFF_VAR : (isConst ? NKB_DIFF_CONST : NKB_DIFF_NONE);
        Check(nkb_op_set_factors(m_h.get(), f.lambda, mode, f.coeffD.data()));
    }
    nkb_op *Handle() const
    {
        return m_h.get();
    }

private:
    B200OpHandle m_h;
};

using BwdTrans_B200        = SingleOutput_B200<eBwdTrans>;
using IProductWRTBase_B200 = SingleOutput_B200<eIProductWRTBase>;
using Helmholtz_B200       = SingleOutput_B200<eHelmholtz>;

// PhysDeriv: three outputs, or one direction (PhysDeriv.cpp:272-)
class PhysDeriv_B200 : public Operator
{
public:
    PhysDeriv_B200(const CollectionData &d, const FactorMap &) : m_h(d, ePhysDeriv)
    {
        m_in    = m_h.m_in;
        m_out   = m_h.m_out;
        m_nelmt = unsigned(d.nelmt);
    }
    void operator()(const Array1D &input, Array1D &o0, Array1D &o1, Array1D &o2,
                    Array1D &) override
    {
        if (input.size() < m_in || o0.size() < m_out || o1.size() < m_out || o2.size() < m_out)
            throw NekError(NKB_ERR_INVALID, "array smaller than the operator's size");
        Check(nkb_op_apply(m_h.get(), input.data(), o0.data(), o1.data(), o2.data(), NKB_HOST_PTRS,
                           nullptr));
    }
    void operator()(int dir, const Array1D &input, Array1D &output, Array1D &wsp) override
    {
        if (dir < 0 || dir > 2)
            throw NekError(NKB_ERR_INVALID, "PhysDeriv direction must be 0, 1 or 2");
        Array1D t[3] = {Array1D(m_out), Array1D(m_out), Array1D(m_out)};
        (*this)(input, t[0], t[1], t[2], wsp);
        output.assign(t[dir].begin(), t[dir].end());
    }

private:
    B200OpHandle m_h;
};

// LinearAdvectionDiffusionReaction (LinearAdvectionDiffusionReaction.cpp:548-790):
// coefficients in and out; UpdateFactors takes lambda (the operator applies
// -lambda), UpdateVarcoeffs the advection velocities (scaled by -1/lambda)
class LinearAdvectionDiffusionReaction_B200 : public Operator
{
public:
    LinearAdvectionDiffusionReaction_B200(const CollectionData &d, const FactorMap &f)
        : m_h(d, eLinearAdvectionDiffusionReaction),
          m_nqtot(size_t(d.nelmt) * size_t(d.nq[0]) * size_t(d.nq[1]) * size_t(d.nq[2]))
    {
        m_in    = m_h.m_in;
        m_out   = m_h.m_out;
        m_nelmt = unsigned(d.nelmt);
        UpdateFactors(f);
    }
    void operator()(const Array1D &input, Array1D &output0, Array1D &, Array1D &,
                    Array1D &) override
    {
        if (input.size() < m_in || output0.size() < m_out)
            throw NekError(NKB_ERR_INVALID, "array smaller than the operator's size");
        Check(nkb_op_apply(m_h.get(), input.data(), output0.data(), nullptr, nullptr,
                           NKB_HOST_PTRS, nullptr));
    }
    void operator()(int, const Array1D &, Array1D &, Array1D &) override
    {
        throw NekError(NKB_ERR_INVALID, "Not valid for this operator.");
    }
    // UpdateFactors (LinearAdvectionDiffusionReaction.cpp:578-590)
    void UpdateFactors(const FactorMap &f) override
    {
        Check(nkb_op_set_factors(m_h.get(), f.lambda, NKB_DIFF_NONE, nullptr));
    }
    // UpdateVarcoeffs (LinearAdvectionDiffusionReaction.cpp:598-723)
    void UpdateVarcoeffs(VarCoeffMap &v) override
    {
        if (v.velx.size() < m_nqtot || v.vely.size() < m_nqtot || v.velz.size() < m_nqtot)
            throw NekError(NKB_ERR_INVALID, "Must define at least one advection velocity");
        Check(nkb_op_set_varcoeffs(m_h.get(), v.velx.data(), v.vely.data(), v.velz.data(),
                                   NKB_HOST_PTRS));
    }

private:
    B200OpHandle m_h;
    size_t m_nqtot; // quadrature points of the collection
};

// IProductWRTDerivBase: the vector field's three components in entry0..2,
// the result in entry3 (IProductWRTDerivBase.cpp:285-318, coordim 3)
class IProductWRTDerivBase_B200 : public Operator
{
public:
    IProductWRTDerivBase_B200(const CollectionData &d, const FactorMap &)
        : m_h(d, eIProductWRTDerivBase)
    {
        m_in    = m_h.m_in / 3; // per component, as GetInputSize reports it
        m_out   = m_h.m_out;
        m_nelmt = unsigned(d.nelmt);
    }
    void operator()(const Array1D &entry0, Array1D &entry1, Array1D &entry2, Array1D &entry3,
                    Array1D &) override
    {
        if (entry0.size() < m_in || entry1.size() < m_in || entry2.size() < m_in ||
            entry3.size() < m_out)
            throw NekError(NKB_ERR_INVALID, "array smaller than the operator's size");
        Check(nkb_op_apply3(m_h.get(), entry0.data(), entry1.data(), entry2.data(), entry3.data(),
                            NKB_HOST_PTRS, nullptr));
    }
    void operator()(int, const Array1D &, Array1D &, Array1D &) override
    {
        throw NekError(NKB_ERR_INVALID, "Not valid for this operator.");
    }

private:
    B200OpHandle m_h;
};

// Registration of eB200 next to eMatrixFree (the reference registers its
// implementations the same way, e.g. Helmholtz.cpp:764-783)
inline bool RegisterB200Operators()
{
    auto &f = GetOperatorFactory();
    for (ShapeType s : {eHexahedron, ePrism, eTetrahedron})
    {
        f.RegisterCreatorFunction(
            OperatorKey(s, eBwdTrans, eB200, false),
            [](const CollectionData &d, const FactorMap &m) {
                return std::make_shared<BwdTrans_B200>(d, m);
            },
            "BwdTrans_B200");
        f.RegisterCreatorFunction(
            OperatorKey(s, eIProductWRTBase, eB200, false),
            [](const CollectionData &d, const FactorMap &m) {
                return std::make_shared<IProductWRTBase_B200>(d, m);
            },
            "IProductWRTBase_B200");
        f.RegisterCreatorFunction(
            OperatorKey(s, ePhysDeriv, eB200, false),
            [](const CollectionData &d, const FactorMap &m) {
                return std::make_shared<PhysDeriv_B200>(d, m);
            },
            "PhysDeriv_B200");
        f.RegisterCreatorFunction(
            OperatorKey(s, eLinearAdvectionDiffusionReaction, eB200, false),
            [](const CollectionData &d, const FactorMap &m) {
                return std::make_shared<LinearAdvectionDiffusionReaction_B200>(d, m);
            },
            "LinearAdvectionDiffusionReaction_B200");
        f.RegisterCreatorFunction(
            OperatorKey(s, eIProductWRTDerivBase, eB200, false),
            [](const CollectionData &d, const FactorMap &m) {
                return std::make_shared<IProductWRTDerivBase_B200>(d, m);
            },
            "IProductWRTDerivBase_B200");
        f.RegisterCreatorFunction(
            OperatorKey(s, eHelmholtz, eB200, false),
            [](const CollectionData &d, const FactorMap &m) {
                return std::make_shared<Helmholtz_B200>(d, m);
            },
            "Helmholtz_B200");
    }
    return true;
}

// GlobalLinSysIterativeFull + PreconditionerDiagonal + NekLinSysIterCG over
// the Helmholtz collections (GlobalLinSysIterativeFull.cpp:96-384).
class GlobalLinSysIterativeFullB200
{
public:
    GlobalLinSysIterativeFullB200(const std::vector<std::shared_ptr<Helmholtz_B200>> &colls,
                                  const std::vector<int> &localToGlobalMap, int nGlobal, int nDir,
                                  const Array1D &sign = Array1D(), int device = 0)
        : m_colls(colls)
    {
        std::vector<nkb_op *> ops;
        long nloc = 0;
        for (auto &c : colls)
        {
            ops.push_back(c->Handle());
            nloc += c->GetInputSize();
        }
        nkb_sys_desc d{};
        d.nops   = int(ops.size());
        d.ops    = ops.data();
        d.nloc   = nloc;
        d.nglob  = nGlobal;
        d.ndir   = nDir;
        d.map    = localToGlobalMap.data();
        d.sign   = sign.empty() ? nullptr : sign.data();
        d.device = device;
        Check(nkb_sys_create(&d, &m_sys));
        m_nloc = nloc;
    }
    ~GlobalLinSysIterativeFullB200()
    {
        nkb_sys_destroy(m_sys);
    }
    // v_Solve(pLocInput, pLocOutput, ...): pLocOutput holds the Dirichlet
    // values on entry and the solution on return. Reaching maxit throws, where
    // the reference prints "WARNING: Exceeded maxIt" (NekLinSysIterCG.cpp:216-231).
    nkb_cg_report Solve(const Array1D &locInput, Array1D &locOutput, double tol = 1e-9,
                        int maxit = 5000)
    {
        if (long(locInput.size()) < m_nloc || long(locOutput.size()) < m_nloc)
            throw NekError(NKB_ERR_INVALID, "local arrays smaller than the system");
        nkb_cg_opts o{};
        o.tol            = tol;
        o.maxit          = maxit;
        o.check_interval = 16;
        o.use_graph      = 1;
        nkb_cg_report r{};
        Check(nkb_cg_solve(m_sys, locInput.data(), locOutput.data(), &o, &r, NKB_HOST_PTRS,
                           nullptr));
        return r;
    }

private:
    std::vector<std::shared_ptr<Helmholtz_B200>> m_colls;
    nkb_sys *m_sys = nullptr;
    long m_nloc    = 0;
};

} // namespace collections
} // namespace nkb
