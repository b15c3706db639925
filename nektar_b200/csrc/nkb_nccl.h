// NCCL entry points used by the sharded solve, resolved at run time from
// libnccl.so.2 (the copy a process has loaded already, e.g. through torch,
// else the system's), so that the library itself neither links NCCL nor
// needs it to load.
#pragma once

#include <nccl.h>

namespace nkb
{
struct NcclApi
{
    decltype(&ncclGetVersion) GetVersion;
    decltype(&ncclGetUniqueId) GetUniqueId;
    decltype(&ncclCommInitRank) CommInitRank;
    decltype(&ncclCommDestroy) CommDestroy;
    decltype(&ncclCommAbort) CommAbort;
    decltype(&ncclCommGetAsyncError) CommGetAsyncError;
    decltype(&ncclGetErrorString) GetErrorString;
    decltype(&ncclAllReduce) AllReduce;
    decltype(&ncclSend) Send;
    decltype(&ncclRecv) Recv;
    decltype(&ncclGroupStart) GroupStart;
    decltype(&ncclGroupEnd) GroupEnd;
};

// the resolved entry points, or nullptr (with the error set) when
// libnccl.so.2 or one of them cannot be found
const NcclApi *Nccl();
} // namespace nkb

struct nkb_comm;

namespace nkb
{
ncclComm_t CommHandle(const nkb_comm *c);
int CommRanks(const nkb_comm *c);
int CommRank(const nkb_comm *c);
int CommDevice(const nkb_comm *c);
} // namespace nkb
