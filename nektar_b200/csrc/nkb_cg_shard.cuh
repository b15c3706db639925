// The CG sharded over element partitions, on the device (included at the end
// of nkb_cg.cu, whose kernels and solve state it shares): the parallel form of
// GlobalLinSysIterativeFull + NekLinSysIterCG that MPI runs of the reference
// use (one partition per rank, MeshPartition.cpp:99; the shared dofs summed
// across partitions by AssemblyMapCG::UniversalAssemble,
// AssemblyMapCG.cpp:2894-2906; the three dot products of an iteration summed
// in one all-reduce, NekLinSysIterCG.cpp:310).
//
// Every shard is an ordinary nkb_sys over its partition's elements whose
// global dofs are numbered
//   [Dirichlet | free, this shard only | free shared, owned | free shared, others']
// so that a dot product counts a free dof on the shard that owns it through
// an index bound (nown), and the partial (s,w) of the assemble is complete
// on the first block (nint). One iteration, per shard:
//   k_update (partials over i < nown), operator (gathered), k_assemble
//   ((s,w) over the first nint free dofs), k_pack (the values each neighbour
//   shares), the exchange, k_unpack (each shared dof = the sum of every
//   sharing shard's value in rank order, so all shards hold the same bits;
//   (s,w) over the owned shared dofs), k_shard_sums (the shard's three sums),
//   the all-reduce of the sums, k_scalars_tot (alpha, beta, convergence).
// The exchange and the all-reduce are NCCL (ncclSend / ncclRecv to every
// neighbour in one group; ncclAllReduce of the sums) when the group has a
// communicator, one shard per process and GPU; without one, all shards live
// in this process on one device and the exchange is device copies between
// their buffers, the all-reduce a fixed-order sum (the sharded recurrence run
// on one GPU). The K iterations between convergence polls are one CUDA graph
// in both cases (NCCL calls captured with the kernels).

#include "nkb_nccl.h"

namespace nkb
{

// buf[k] = v[idx[k]]
__global__ void k_pack(int n, const int *__restrict__ idx, const double *__restrict__ v,
                       double *__restrict__ buf, const CGState *st)
{
    if (st && st->done)
        return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        buf[k] = v[idx[k]];
}

// v[shared[k]] = sum over the sharing shards in rank order (src -1: this
// shard's own value, else a position in recv); partial (v,w) over the owned
// shared free dofs ndir + nint <= g < ndir + nown
__global__ void k_unpack(int n, const int *__restrict__ shared, const int *__restrict__ sptr,
                         const int *__restrict__ ssrc, const double *__restrict__ recv,
                         double *__restrict__ v, int ndir, int nint, int nown,
                         const double *__restrict__ w, const CGState *st, double *part)
{
    if (st && st->done)
        return;
    double sw = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    {
        const int g    = shared[k];
        const double o = v[g];
        double acc     = 0.0;
        for (int c = sptr[k]; c < sptr[k + 1]; ++c)
        {
            const int src = ssrc[c];
            acc += src < 0 ? o : recv[src];
        }
        v[g] = acc;
        if (w && g - ndir >= nint && g - ndir < nown)
            sw += acc * w[g];
    }
    if (part)
        BlockSum2(sw, 0.0, part);
}

// the shard's sums: (a0, a1, b0) = (partA[0], partA[1], partB[0] + partD[0])
__global__ void k_shard_sums(const double *partA, int nbA, const double *partB, int nbB,
                             const double *partD, int nbD, double *sums)
{
    const double a0 = ReducePart(partA, nbA, 0);
    const double a1 = ReducePart(partA, nbA, 1);
    double b0       = ReducePart(partB, nbB, 0);
    if (nbD)
        b0 += ReducePart(partD, nbD, 0);
    if (threadIdx.x == 0)
    {
        sums[0] = a0;
        sums[1] = a1;
        sums[2] = b0;
        sums[3] = 0.0;
    }
}

// the group's totals over n shards' sums, in rank order
__global__ void k_group_total(const double *sums, int n, double *tot)
{
    if (threadIdx.x < 4)
    {
        double t = 0.0;
        for (int i = 0; i < n; ++i)
            t += sums[4 * i + threadIdx.x];
        tot[threadIdx.x] = t;
    }
}

__global__ void k_scalars_tot(CGState *st, const double *tot, int mode)
{
    if (st->done)
        return;
    ScalarStep(st, tot[0], tot[1], tot[2], mode);
}

struct ShardDev
{
    nkb_sys *S = nullptr;
    int rank = 0, nint = 0, nown = 0, nshared = 0, nnbr = 0;
    std::vector<int> nbr, nptr; // host copies
    int *d_shared = nullptr, *d_sptr = nullptr, *d_ssrc = nullptr, *d_nidx = nullptr;
    unsigned char *d_dcnt = nullptr;
    double *send = nullptr, *recv = nullptr, *partD = nullptr, *sums = nullptr;
    int nbuf = 0;
    const double *db = nullptr; // this solve's device b_loc
    double *dx = nullptr;       // this solve's device x_loc
};
} // namespace nkb

struct nkb_shard_group
{
    std::vector<nkb::ShardDev> sh;
    nkb_comm *comm = nullptr;
    int nranks = 0, device = 0;
    cudaStream_t s = nullptr;
    double *gsums = nullptr, *tot = nullptr; // [shards][4], [4]
    cudaGraphExec_t graph = nullptr;
    int graph_k = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    CGState *h_st = nullptr; // pinned
    long launches = 0;
};

namespace nkb
{
static void FreeShard(ShardDev &d)
{
    for (void *p : {(void *)d.d_shared, (void *)d.d_sptr, (void *)d.d_ssrc, (void *)d.d_nidx,
                    (void *)d.d_dcnt, (void *)d.send, (void *)d.recv, (void *)d.partD,
                    (void *)d.sums})
        cudaFree(p);
}

static void ReleaseGroup(nkb_shard_group *G)
{
    cudaSetDevice(G->device);
    if (G->s)
        cudaStreamSynchronize(G->s);
    if (G->graph)
        cudaGraphExecDestroy(G->graph);
    for (ShardDev &d : G->sh)
    {
        FreeShard(d);
        if (d.S)
            d.S->sv = SolveCtx(); // its solves ran on the group's stream
    }
    cudaFree(G->gsums);
    cudaFree(G->tot);
    if (G->h_st)
        cudaFreeHost(G->h_st);
    if (G->ev0)
        cudaEventDestroy(G->ev0);
    if (G->ev1)
        cudaEventDestroy(G->ev1);
    if (G->s)
        cudaStreamDestroy(G->s);
    delete G;
}

// v (each shard's global vector, chosen by `which`) summed over the shards
// at the shared dofs; with `partial`, the owned shared part of (v, w) goes to
// each shard's partD. skip_done: the kernels do nothing once converged.
static int Exchange(nkb_shard_group *G, double *nkb_sys::*which, bool partial, bool skip_done)
{
    cudaStream_t s = G->s;
    for (ShardDev &d : G->sh)
        if (d.nbuf)
        {
            k_pack<<<Blocks(d.nbuf), kRedThreads, 0, s>>>(d.nbuf, d.d_nidx, d.S->*which, d.send,
                                                          skip_done ? d.S->st : nullptr);
            ++G->launches;
        }
    if (G->comm)
    {
        const ShardDev &d = G->sh[0];
        const NcclApi *n  = Nccl();
        ncclComm_t c      = CommHandle(G->comm);
        ncclResult_t r    = n->GroupStart();
        for (int k = 0; k < d.nnbr && r == ncclSuccess; ++k)
        {
            const size_t len = size_t(d.nptr[k + 1] - d.nptr[k]);
            r = n->Send(d.send + d.nptr[k], len, ncclFloat64, d.nbr[k], c, s);
            if (r == ncclSuccess)
                r = n->Recv(d.recv + d.nptr[k], len, ncclFloat64, d.nbr[k], c, s);
        }
        const ncclResult_t r2 = n->GroupEnd();
        if (r != ncclSuccess || r2 != ncclSuccess)
            return SetError(NKB_ERR_CUDA, "sharded exchange: %s",
                            n->GetErrorString(r != ncclSuccess ? r : r2));
    }
    else
        for (ShardDev &d : G->sh)
            for (int k = 0; k < d.nnbr; ++k)
            {
                const ShardDev &q = G->sh[d.nbr[k]];
                int kk            = 0;
                while (q.nbr[kk] != d.rank)
                    ++kk;
                NKB_CUDA_TRY(cudaMemcpyAsync(d.recv + d.nptr[k], q.send + q.nptr[kk],
                                             size_t(d.nptr[k + 1] - d.nptr[k]) * sizeof(double),
                                             cudaMemcpyDeviceToDevice, s));
            }
    for (ShardDev &d : G->sh)
    {
        nkb_sys *S = d.S;
        if (d.nshared)
        {
            k_unpack<<<Blocks(d.nshared), kRedThreads, 0, s>>>(
                d.nshared, d.d_shared, d.d_sptr, d.d_ssrc, d.recv, S->*which, S->ndir, d.nint,
                d.nown, partial ? S->w : nullptr, skip_done ? S->st : nullptr,
                partial ? d.partD : nullptr);
            ++G->launches;
        }
        else if (partial)
            NKB_CUDA_TRY(cudaMemsetAsync(d.partD, 0, 2 * sizeof(double), s));
    }
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

static int PartDBlocks(const ShardDev &d)
{
    return d.nshared ? Blocks(d.nshared) : 1;
}

// every shard's sums, their total over the group, the scalar step. After
// k_init (mode 0) partA holds (b,b), (r,r) over Blocks(nglob) CTAs and serves
// as partB too; after k_precon / k_update partA has Blocks(nn) CTAs, partB
// (k_assemble) Blocks(nglob) and partD (k_unpack) the owned shared part of
// (s,w).
static int Scalars(nkb_shard_group *G, int mode)
{
    cudaStream_t s = G->s;
    for (size_t i = 0; i < G->sh.size(); ++i)
    {
        ShardDev &d = G->sh[i];
        nkb_sys *S  = d.S;
        double *out = G->comm ? d.sums : G->gsums + 4 * i;
        if (mode == 0)
            k_shard_sums<<<1, 1024, 0, s>>>(S->partA, Blocks(S->nglob), S->partA, Blocks(S->nglob),
                                            nullptr, 0, out);
        else
            k_shard_sums<<<1, 1024, 0, s>>>(S->partA, Blocks(S->nn), S->partB, Blocks(S->nglob),
                                            d.partD, PartDBlocks(d), out);
        ++G->launches;
    }
    if (G->comm)
    {
        const NcclApi *n     = Nccl();
        const ncclResult_t r = n->AllReduce(G->sh[0].sums, G->tot, 4, ncclFloat64, ncclSum,
                                            CommHandle(G->comm), s);
        if (r != ncclSuccess)
            return SetError(NKB_ERR_CUDA, "sharded all-reduce: %s", n->GetErrorString(r));
    }
    else
    {
        k_group_total<<<1, 32, 0, s>>>(G->gsums, int(G->sh.size()), G->tot);
        ++G->launches;
    }
    for (ShardDev &d : G->sh)
    {
        k_scalars_tot<<<1, 1, 0, s>>>(d.S->st, G->tot, mode);
        ++G->launches;
    }
    NKB_CUDA_TRY(cudaGetLastError());
    return NKB_OK;
}

static int GroupIteration(nkb_shard_group *G)
{
    cudaStream_t s = G->s;
    for (ShardDev &d : G->sh)
    {
        nkb_sys *S = d.S;
        k_update<double><<<Blocks(S->nn), kRedThreads, 0, s>>>(S->nn, S->ndir, S->st, S->p, S->q,
                                                               S->x, S->r, S->w, S->s, S->d_dinv,
                                                               S->partA, d.nown, 1);
        int rc = Matvec(S, S->w, S->yl, true, s, &S->st->done);
        if (rc)
            return rc;
        k_assemble<double><<<Blocks(S->nglob), kRedThreads, 0, s>>>(
            S->nglob, S->ndir, S->d_aptr, S->d_aidx, S->d_sign, S->yl, S->s, S->w, S->st, S->partB,
            d.nint);
        G->launches += 2 + long(S->ops.size());
    }
    int rc = Exchange(G, &nkb_sys::s, true, true);
    if (rc)
        return rc;
    return Scalars(G, 2);
}

static int EnsureGroupGraph(nkb_shard_group *G, int K)
{
    if (G->graph && G->graph_k == K)
        return NKB_OK;
    if (G->graph)
        cudaGraphExecDestroy(G->graph);
    G->graph         = nullptr;
    const long saved = G->launches;
    cudaGraph_t g;
    NKB_CUDA_TRY(cudaStreamBeginCapture(G->s, cudaStreamCaptureModeThreadLocal));
    int crc = NKB_OK;
    for (int k = 0; k < K && !crc; ++k)
        crc = GroupIteration(G);
    cudaError_t ce = cudaStreamEndCapture(G->s, &g);
    G->launches    = saved;
    if (crc)
        return crc;
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "sharded CG graph capture: %s", cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&G->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess)
        return SetError(NKB_ERR_CUDA, "sharded CG graph instantiate: %s", cudaGetErrorString(ce));
    G->graph_k = K;
    return NKB_OK;
}

// one shard's plan against its system; host arrays
static int CheckPlan(const nkb_sys *S, const nkb_shard_plan &p, int nranks)
{
    if (p.rank < 0 || p.rank >= nranks || p.nint < 0 || p.nown < p.nint || p.nown > S->nn ||
        p.nshared < 0 || p.nnbr < 0 || p.nnbr >= nranks ||
        (p.nshared && (!p.shared || !p.sptr || !p.ssrc)) ||
        (p.nnbr && (!p.nbr || !p.nptr || !p.nidx)))
        return SetError(NKB_ERR_INVALID, "shard %d: bad plan sizes", p.rank);
    if (p.nnbr && p.nptr[0] != 0)
        return SetError(NKB_ERR_INVALID, "shard %d: nptr[0] != 0", p.rank);
    for (int k = 0; k < p.nnbr; ++k)
        if (p.nptr[k + 1] <= p.nptr[k] || p.nbr[k] < 0 || p.nbr[k] >= nranks ||
            p.nbr[k] == p.rank || (k && p.nbr[k] <= p.nbr[k - 1]))
            return SetError(NKB_ERR_INVALID, "shard %d: neighbour %d of the plan", p.rank, k);
    const int nbuf = p.nnbr ? p.nptr[p.nnbr] : 0;
    for (int t = 0; t < nbuf; ++t)
        if (p.nidx[t] < 0 || p.nidx[t] >= S->nglob)
            return SetError(NKB_ERR_INVALID, "shard %d: nidx[%d] = %d outside [0,%d)", p.rank, t,
                            p.nidx[t], S->nglob);
    if (p.nshared && p.sptr[0] != 0)
        return SetError(NKB_ERR_INVALID, "shard %d: sptr[0] != 0", p.rank);
    std::vector<char> seen(S->nglob, 0);
    for (int k = 0; k < p.nshared; ++k)
    {
        const int g = p.shared[k];
        if (g < 0 || g >= S->nglob || seen[g]++ || (g >= S->ndir && g - S->ndir < p.nint))
            return SetError(NKB_ERR_INVALID, "shard %d: shared dof %d", p.rank, g);
        if (p.sptr[k + 1] < p.sptr[k] + 2)
            return SetError(NKB_ERR_INVALID, "shard %d: shared dof %d has fewer than two sources",
                            p.rank, g);
        int own = 0;
        for (int c = p.sptr[k]; c < p.sptr[k + 1]; ++c)
        {
            if (p.ssrc[c] < -1 || p.ssrc[c] >= nbuf)
                return SetError(NKB_ERR_INVALID, "shard %d: source %d of shared dof %d", p.rank,
                                p.ssrc[c], g);
            own += p.ssrc[c] == -1;
        }
        if (own != 1)
            return SetError(NKB_ERR_INVALID, "shard %d: shared dof %d lists its own value %d times",
                            p.rank, g, own);
    }
    for (int g = S->ndir + p.nint; g < S->nglob; ++g)
        if (!seen[g])
            return SetError(NKB_ERR_INVALID, "shard %d: free dof %d past nint is not shared",
                            p.rank, g);
    return NKB_OK;
}

static int UploadPlan(ShardDev &d, const nkb_shard_plan &p, int ndir)
{
    auto up = [](void **dst, const void *src, size_t bytes) -> bool {
        if (!bytes)
            return true;
        return cudaMalloc(dst, bytes) == cudaSuccess &&
               cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
    };
    d.rank    = p.rank;
    d.nint    = p.nint;
    d.nown    = p.nown;
    d.nshared = p.nshared;
    d.nnbr    = p.nnbr;
    d.nbr.assign(p.nbr, p.nbr + p.nnbr);
    if (p.nnbr)
        d.nptr.assign(p.nptr, p.nptr + p.nnbr + 1);
    d.nbuf             = p.nnbr ? p.nptr[p.nnbr] : 0;
    const int ncontrib = p.nshared ? p.sptr[p.nshared] : 0;
    std::vector<unsigned char> dcnt(std::max(ndir, 1), 1);
    if (p.dir_owned)
        for (int g = 0; g < ndir; ++g)
            dcnt[g] = p.dir_owned[g] ? 1 : 0;
    const bool ok =
        up((void **)&d.d_shared, p.shared, size_t(p.nshared) * sizeof(int)) &&
        up((void **)&d.d_sptr, p.sptr, p.nshared ? size_t(p.nshared + 1) * sizeof(int) : 0) &&
        up((void **)&d.d_ssrc, p.ssrc, size_t(ncontrib) * sizeof(int)) &&
        up((void **)&d.d_nidx, p.nidx, size_t(d.nbuf) * sizeof(int)) &&
        up((void **)&d.d_dcnt, dcnt.data(), dcnt.size()) &&
        cudaMalloc(&d.send, std::max<size_t>(d.nbuf, 1) * sizeof(double)) == cudaSuccess &&
        cudaMalloc(&d.recv, std::max<size_t>(d.nbuf, 1) * sizeof(double)) == cudaSuccess &&
        cudaMalloc(&d.partD, 2 * size_t(kRedBlocks) * sizeof(double)) == cudaSuccess &&
        cudaMalloc(&d.sums, 4 * sizeof(double)) == cudaSuccess;
    if (!ok)
        return SetError(NKB_ERR_NOMEM, "shard %d: plan upload", p.rank);
    return NKB_OK;
}
} // namespace nkb

extern "C" int nkb_shard_group_create(nkb_sys *const *systems, const nkb_shard_plan *plans,
                                      int nlocal, nkb_comm *comm, nkb_shard_group **out)
{
    ClearError();
    if (!systems || !plans || nlocal < 1 || !out)
        return SetError(NKB_ERR_INVALID, "nkb_shard_group_create: bad arguments");
    *out         = nullptr;
    const int nr = comm ? CommRanks(comm) : nlocal;
    if (comm && nlocal != 1)
        return SetError(NKB_ERR_INVALID, "nkb_shard_group_create: one shard per communicator rank");
    if (comm && plans[0].rank != CommRank(comm))
        return SetError(NKB_ERR_INVALID,
                        "nkb_shard_group_create: plan rank %d != communicator rank %d",
                        plans[0].rank, CommRank(comm));
    if (!systems[0])
        return SetError(NKB_ERR_INVALID, "nkb_shard_group_create: NULL system 0");
    const int device = systems[0]->device;
    for (int i = 0; i < nlocal; ++i)
    {
        const nkb_sys *S = systems[i];
        if (!S)
            return SetError(NKB_ERR_INVALID, "nkb_shard_group_create: NULL system %d", i);
        if (!comm && plans[i].rank != i)
            return SetError(NKB_ERR_INVALID, "nkb_shard_group_create: the plans of a group "
                                             "without a communicator are ranks 0..%d in order",
                            nlocal - 1);
        if (S->device != device || (comm && CommDevice(comm) != device))
            return SetError(NKB_ERR_INVALID, "nkb_shard_group_create: shards on different devices");
        if (Busy(S) || S->sh->grouped || S->sh.use_count() > 1 || S->sh->nblk)
            return SetError(NKB_ERR_INVALID, "nkb_shard_group_create: system %d is busy, cloned, "
                                             "in a group or block-preconditioned",
                            i);
        for (int j = 0; j < i; ++j)
            if (systems[j] == S)
                return SetError(NKB_ERR_INVALID, "nkb_shard_group_create: system %d given twice",
                                i);
        if (int rc = CheckPlan(S, plans[i], nr))
            return rc;
    }
    // the lists of two shards in one process must agree
    if (!comm)
        for (int i = 0; i < nlocal; ++i)
            for (int k = 0; k < plans[i].nnbr; ++k)
            {
                const nkb_shard_plan &q = plans[plans[i].nbr[k]];
                int kk                  = 0;
                while (kk < q.nnbr && q.nbr[kk] != i)
                    ++kk;
                if (kk == q.nnbr ||
                    q.nptr[kk + 1] - q.nptr[kk] != plans[i].nptr[k + 1] - plans[i].nptr[k])
                    return SetError(NKB_ERR_INVALID, "nkb_shard_group_create: shards %d and %d "
                                                     "disagree on their shared dofs",
                                    i, plans[i].nbr[k]);
            }
    for (int i = 0; i < nlocal; ++i)
        if (!systems[i]->sh->d_dM)
            return SetError(NKB_ERR_UNSUPPORTED, "nkb_shard_group_create: shard %d has operators "
                                                 "with different lambdas",
                            i);
    NKB_CUDA_TRY(cudaSetDevice(device));
    nkb_shard_group *G = new nkb_shard_group();
    G->comm            = comm;
    G->nranks          = nr;
    G->device          = device;
    G->sh.resize(nlocal);
    auto fail = [&](int code) {
        ReleaseGroup(G);
        return code;
    };
    if (cudaStreamCreateWithFlags(&G->s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&G->ev0) != cudaSuccess || cudaEventCreate(&G->ev1) != cudaSuccess ||
        cudaMalloc(&G->gsums, 4 * size_t(nlocal) * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&G->tot, 4 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&G->h_st, sizeof(CGState)) != cudaSuccess)
        return fail(SetError(NKB_ERR_NOMEM, "nkb_shard_group_create: group buffers"));
    for (int i = 0; i < nlocal; ++i)
    {
        G->sh[i].S = systems[i];
        if (int rc = UploadPlan(G->sh[i], plans[i], systems[i]->ndir))
            return fail(rc);
    }
    // the Jacobi diagonal of the whole mesh: the shards' assembled mass and
    // Laplacian parts summed at the shared dofs, then recombined
    for (double *SysShared::*part : {&SysShared::d_dM, &SysShared::d_dL})
    {
        for (ShardDev &d : G->sh)
            if (cudaMemcpyAsync(d.S->bglob, d.S->sh.get()->*part, d.S->nglob * sizeof(double),
                                cudaMemcpyDeviceToDevice, G->s) != cudaSuccess)
                return fail(SetError(NKB_ERR_CUDA, "nkb_shard_group_create: diagonal copy"));
        if (int rc = Exchange(G, &nkb_sys::bglob, false, false))
            return fail(rc);
        for (ShardDev &d : G->sh)
            if (cudaMemcpyAsync(d.S->sh.get()->*part, d.S->bglob, d.S->nglob * sizeof(double),
                                cudaMemcpyDeviceToDevice, G->s) != cudaSuccess)
                return fail(SetError(NKB_ERR_CUDA, "nkb_shard_group_create: diagonal copy"));
    }
    for (ShardDev &d : G->sh)
    {
        nkb_sys *S          = d.S;
        const double lambda = S->has_lambda ? S->lambda : S->ops[0]->lambda;
        k_combine_dinv<<<Blocks(S->nn), kRedThreads, 0, G->s>>>(S->nn, S->ndir, lambda,
                                                                S->sh->d_dM, S->sh->d_dL,
                                                                S->d_dinv, S->dinv32);
    }
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(G->s) != cudaSuccess)
        return fail(SetError(NKB_ERR_CUDA, "nkb_shard_group_create: Jacobi diagonal"));
    for (ShardDev &d : G->sh)
        d.S->sh->grouped = true;
    *out = G;
    return NKB_OK;
}

extern "C" int nkb_shard_group_solve(nkb_shard_group *G, const double *const *b_locs,
                                     double *const *x_locs, const nkb_cg_opts *opts,
                                     nkb_cg_report *reps, int flags)
{
    ClearError();
    if (!G || !b_locs || !x_locs)
        return SetError(NKB_ERR_INVALID, "nkb_shard_group_solve: NULL argument");
    nkb_cg_opts o;
    std::memset(&o, 0, sizeof(o));
    o.tol            = 1e-9;
    o.maxit          = 5000;
    o.check_interval = 16;
    o.use_graph      = 1;
    if (opts)
        o = *opts;
    if (o.tol <= 0)
        o.tol = 1e-9;
    if (o.maxit <= 0)
        o.maxit = 5000;
    if (o.check_interval <= 0)
        o.check_interval = 16;
    if (o.mixed)
        return SetError(NKB_ERR_UNSUPPORTED, "nkb_shard_group_solve: FP64 only");
    NKB_CUDA_TRY(cudaSetDevice(G->device));
    cudaStream_t s = G->s;
    G->launches    = 0;
    for (size_t i = 0; i < G->sh.size(); ++i)
    {
        ShardDev &d = G->sh[i];
        nkb_sys *S  = d.S;
        if (!b_locs[i] || !x_locs[i])
            return SetError(NKB_ERR_INVALID, "nkb_shard_group_solve: NULL vector of shard %d",
                            d.rank);
        S->sv   = SolveCtx();
        S->sv.o = o;
        S->sv.s = s;
        d.db    = b_locs[i];
        d.dx    = x_locs[i];
        if (flags & NKB_HOST_PTRS)
        {
            if (!S->stage)
            {
                if (cudaMalloc(&S->stage, 2 * S->nloc * sizeof(double)) != cudaSuccess)
                    return SetError(NKB_ERR_NOMEM, "nkb_shard_group_solve: staging buffers");
                S->bytes += 2 * S->nloc * sizeof(double);
            }
            NKB_CUDA_TRY(cudaMemcpyAsync(S->stage, b_locs[i], S->nloc * sizeof(double),
                                         cudaMemcpyHostToDevice, s));
            NKB_CUDA_TRY(cudaMemcpyAsync(S->stage + S->nloc, x_locs[i], S->nloc * sizeof(double),
                                         cudaMemcpyHostToDevice, s));
            d.db = S->stage;
            d.dx = S->stage + S->nloc;
        }
    }
    NKB_CUDA_TRY(cudaEventRecord(G->ev0, s));
    // Dirichlet lifting (GlobalLinSysIterativeFull.cpp:104-164) and the
    // assembled right-hand side, summed at the shared dofs
    for (ShardDev &d : G->sh)
    {
        nkb_sys *S = d.S;
        if (int rc = ResetState(S))
            return rc;
        if (int rc = Matvec(S, d.dx, S->yl, false, s))
            return rc;
        k_sub_loc<<<Blocks(S->nloc), kRedThreads, 0, s>>>(S->nloc, d.db, S->yl, S->tl);
        k_assemble<double><<<Blocks(S->nglob), kRedThreads, 0, s>>>(
            S->nglob, S->ndir, S->d_aptr, S->d_aidx, S->d_sign, S->tl, S->bglob, nullptr, nullptr,
            nullptr, S->nn);
        G->launches += 2 + long(S->ops.size());
    }
    if (int rc = Exchange(G, &nkb_sys::bglob, false, false))
        return rc;
    for (ShardDev &d : G->sh)
    {
        nkb_sys *S = d.S;
        k_init<<<Blocks(S->nglob), kRedThreads, 0, s>>>(S->nglob, S->ndir, S->bglob, S->r, S->x,
                                                        S->w, S->s, S->p, S->q, S->partA, d.d_dcnt,
                                                        d.nown);
        ++G->launches;
    }
    if (int rc = Scalars(G, 0))
        return rc;
    // the first direction
    for (ShardDev &d : G->sh)
    {
        nkb_sys *S = d.S;
        k_precon<double><<<Blocks(S->nn), kRedThreads, 0, s>>>(S->nn, S->ndir, S->st, S->r, S->w,
                                                               S->d_dinv, S->partA, d.nown);
        if (int rc = Matvec(S, S->w, S->yl, true, s, &S->st->done))
            return rc;
        k_assemble<double><<<Blocks(S->nglob), kRedThreads, 0, s>>>(
            S->nglob, S->ndir, S->d_aptr, S->d_aidx, S->d_sign, S->yl, S->s, S->w, S->st, S->partB,
            d.nint);
        G->launches += 2 + long(S->ops.size());
    }
    if (int rc = Exchange(G, &nkb_sys::s, true, true))
        return rc;
    if (int rc = Scalars(G, 1))
        return rc;
    const bool use_graph = o.use_graph != 0;
    long per_iter        = G->comm ? 0 : 1;
    for (const ShardDev &d : G->sh)
        per_iter += 4 + long(d.S->ops.size()) + (d.nbuf ? 1 : 0) + (d.nshared ? 1 : 0);
    if (use_graph)
        if (int rc = EnsureGroupGraph(G, o.check_interval))
            return rc;
    const int max_passes = o.maxit / o.check_interval + 2;
    nkb_sys *S0          = G->sh[0].S;
    for (int pass = 0;; ++pass)
    {
        NKB_CUDA_TRY(cudaMemcpyAsync(G->h_st, S0->st, sizeof(CGState), cudaMemcpyDeviceToHost, s));
        NKB_CUDA_TRY(cudaStreamSynchronize(s));
        if (G->h_st->done || pass >= max_passes)
            break;
        if (use_graph)
        {
            NKB_CUDA_TRY(cudaGraphLaunch(G->graph, s));
            G->launches += long(o.check_interval) * per_iter;
        }
        else
            for (int k = 0; k < o.check_interval; ++k)
                if (int rc = GroupIteration(G))
                    return rc;
    }
    // x_loc += GlobalToLocal(x) on every shard
    for (ShardDev &d : G->sh)
    {
        nkb_sys *S = d.S;
        k_global_to_local<<<Blocks(S->nloc), kRedThreads, 0, s>>>(S->nloc, S->d_map, S->d_sign,
                                                                   S->x, S->tl);
        k_axpy_loc<<<Blocks(S->nloc), kRedThreads, 0, s>>>(S->nloc, 1.0, S->tl, d.dx);
        G->launches += 2;
    }
    NKB_CUDA_TRY(cudaEventRecord(G->ev1, s));
    if (flags & NKB_HOST_PTRS)
        for (size_t i = 0; i < G->sh.size(); ++i)
            NKB_CUDA_TRY(cudaMemcpyAsync(x_locs[i], G->sh[i].dx,
                                         G->sh[i].S->nloc * sizeof(double),
                                         cudaMemcpyDeviceToHost, s));
    NKB_CUDA_TRY(cudaMemcpyAsync(G->h_st, S0->st, sizeof(CGState), cudaMemcpyDeviceToHost, s));
    NKB_CUDA_TRY(cudaStreamSynchronize(s));
    for (ShardDev &d : G->sh)
        d.S->sv = SolveCtx();
    const CGState h = *G->h_st;
    float ms        = 0.f;
    cudaEventElapsedTime(&ms, G->ev0, G->ev1);
    if (reps)
        for (size_t i = 0; i < G->sh.size(); ++i)
        {
            nkb_cg_report &rep = reps[i];
            std::memset(&rep, 0, sizeof(rep));
            rep.iterations      = h.iter;
            rep.rel_residual    = std::sqrt(h.eps / h.rhs_mag);
            rep.converged       = (h.done && h.status == NKB_OK) ? 1 : 0;
            rep.device_ms       = ms;
            rep.kernel_launches = G->launches;
        }
    for (ShardDev &d : G->sh)
        for (nkb_op *op : d.S->ops)
            if (int rc = CheckOpError(op))
                return rc;
    if (h.status == NKB_ERR_NONFINITE)
        return SetError(NKB_ERR_NONFINITE,
                        "nkb_shard_group_solve: non-finite CG scalar at iteration %d", h.iter);
    if (h.status == NKB_ERR_NOT_CONVERGED || !h.done)
        return SetError(NKB_ERR_NOT_CONVERGED,
                        "nkb_shard_group_solve: CG iterations made = %d exceeded maxit (error = %g)",
                        h.iter, std::sqrt(h.eps / h.rhs_mag));
    return NKB_OK;
}

extern "C" void nkb_shard_group_destroy(nkb_shard_group *G)
{
    if (G)
        ReleaseGroup(G);
}
