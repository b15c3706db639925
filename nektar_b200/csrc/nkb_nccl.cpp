// Run-time binding of NCCL and the communicator of the sharded solve
// (nkb_comm_*): one rank per GPU, created from a unique id that rank 0 makes
// and the caller distributes (the reference's ranks share an MPI
// communicator instead; its collectives are those of Comm, used by
// AssemblyMapCG::UniversalAssemble and NekLinSysIterCG).
#include "nkb_internal.h"
#include "nkb_nccl.h"

#include <cuda_runtime.h>
#include <dlfcn.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>

namespace nkb
{
const NcclApi *Nccl()
{
    static std::once_flag once;
    static NcclApi api;
    static bool ok = false;
    static char why[256];
    std::call_once(once, [] {
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h)
        {
            std::snprintf(why, sizeof(why), "libnccl.so.2 not found (%s)", dlerror());
            return;
        }
        bool all = true;
        auto sym = [&](auto &fn, const char *name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
            if (!fn && all)
            {
                std::snprintf(why, sizeof(why), "libnccl.so.2 lacks %s", name);
                all = false;
            }
        };
        sym(api.GetVersion, "ncclGetVersion");
        sym(api.GetUniqueId, "ncclGetUniqueId");
        sym(api.CommInitRank, "ncclCommInitRank");
        sym(api.CommDestroy, "ncclCommDestroy");
        sym(api.CommAbort, "ncclCommAbort");
        sym(api.CommGetAsyncError, "ncclCommGetAsyncError");
        sym(api.GetErrorString, "ncclGetErrorString");
        sym(api.AllReduce, "ncclAllReduce");
        sym(api.Send, "ncclSend");
        sym(api.Recv, "ncclRecv");
        sym(api.GroupStart, "ncclGroupStart");
        sym(api.GroupEnd, "ncclGroupEnd");
        ok = all;
    });
    if (!ok)
    {
        SetError(NKB_ERR_UNSUPPORTED, "NCCL: %s", why);
        return nullptr;
    }
    return &api;
}
} // namespace nkb

using namespace nkb;

struct nkb_comm
{
    ncclComm_t comm = nullptr;
    int nranks = 0, rank = 0, device = 0;
};

extern "C" int nkb_comm_unique_id(unsigned char *id)
{
    ClearError();
    if (!id)
        return SetError(NKB_ERR_INVALID, "nkb_comm_unique_id: NULL id");
    const NcclApi *n = Nccl();
    if (!n)
        return NKB_ERR_UNSUPPORTED;
    ncclUniqueId u;
    const ncclResult_t r = n->GetUniqueId(&u);
    if (r != ncclSuccess)
        return SetError(NKB_ERR_CUDA, "ncclGetUniqueId: %s", n->GetErrorString(r));
    std::memcpy(id, u.internal, NCCL_UNIQUE_ID_BYTES);
    return NKB_OK;
}

extern "C" int nkb_comm_create(const unsigned char *id, int nranks, int rank, int device,
                               nkb_comm **out)
{
    ClearError();
    if (!id || !out || nranks < 1 || rank < 0 || rank >= nranks)
        return SetError(NKB_ERR_INVALID, "nkb_comm_create: bad arguments");
    *out = nullptr;
    const NcclApi *n = Nccl();
    if (!n)
        return NKB_ERR_UNSUPPORTED;
    NKB_CUDA_TRY(cudaSetDevice(device));
    ncclUniqueId u;
    std::memcpy(u.internal, id, NCCL_UNIQUE_ID_BYTES);
    nkb_comm *c = new nkb_comm();
    const ncclResult_t r = n->CommInitRank(&c->comm, nranks, u, rank);
    if (r != ncclSuccess)
    {
        delete c;
        return SetError(NKB_ERR_CUDA, "ncclCommInitRank: %s", n->GetErrorString(r));
    }
    c->nranks = nranks;
    c->rank   = rank;
    c->device = device;
    *out      = c;
    return NKB_OK;
}

extern "C" void nkb_comm_destroy(nkb_comm *c)
{
    if (!c)
        return;
    if (const NcclApi *n = Nccl())
    {
        cudaSetDevice(c->device);
        n->CommDestroy(c->comm);
    }
    delete c;
}

namespace nkb
{
ncclComm_t CommHandle(const nkb_comm *c)
{
    return c->comm;
}
int CommRanks(const nkb_comm *c)
{
    return c->nranks;
}
int CommRank(const nkb_comm *c)
{
    return c->rank;
}
int CommDevice(const nkb_comm *c)
{
    return c->device;
}
} // namespace nkb
