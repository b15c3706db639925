// Batched application of many collections' operators in one call: the loop
// of ExpList::GeneralMatrixOp over the collections of an expansion list
// (MultiRegions/ExpList.cpp:2666-2757, Collection::ApplyOperator per
// collection, Collections/Collection.h:148-189), for meshes that mix shapes
// and orders (one collection per basis key).
//
// On the device the collections are independent kernels of very different
// sizes. They are spread over a few streams, largest first, each to the
// stream with the least work so far (longest-processing-time order), and the
// fork / launches / join sequence is captured once as a CUDA graph, so one
// graph launch runs every collection with the small ones filling the GPU
// beside the large ones. Inputs and outputs are the concatenated per-collection
// local vectors (collection order), as the reference's running offsets give.
#include "nkb_internal.h"
#include "nkb_op.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

using namespace nkb;

struct nkb_batch
{
    int device    = 0;
    int precision = NKB_FP64; // of every operator in the batch
    std::vector<nkb_op *> ops;
    std::vector<long> in_off, out_off;
    long in_size = 0, out_size = 0;
    int nout = 1; // outputs per operator (3 for PhysDeriv)
    std::vector<cudaStream_t> streams;
    std::vector<int> stream_of;  // stream of each operator
    std::vector<int> order;      // launch order (largest first)
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr, order_ev = nullptr;
    cudaStream_t own = nullptr; // used when the caller passes the legacy stream
    cudaGraphExec_t graph = nullptr;
    const void *g_in = nullptr;
    void *g_out = nullptr;
    double *stage = nullptr; // host-pointer staging (in + out)
    float last_ms = 0.f;
};

namespace
{
// work estimate of one collection: bytes of geometry and vectors it moves
double Cost(const nkb_op *op)
{
    const double comps = op->ncomp > 0 ? op->ncomp : 1;
    long in = 0, out = 0;
    nkb_op_sizes(op, &in, &out);
    const double nouts = op->optype == NKB_PHYSDERIV ? 3.0 : 1.0;
    return double(op->nelmt) * comps * op->nt + double(in) + nouts * double(out);
}

template <typename T> int LaunchAll(nkb_batch *B, const T *in, T *out, cudaStream_t s)
{
    NKB_CUDA_TRY(cudaEventRecord(B->fork, s));
    for (cudaStream_t w : B->streams)
        NKB_CUDA_TRY(cudaStreamWaitEvent(w, B->fork, 0));
    for (int c : B->order)
    {
        const nkb_op *op = B->ops[c];
        T *o             = out + B->out_off[c];
        const long no    = long(op->nelmt) * (op->optype == NKB_PHYSDERIV ? op->nt : 0);
        int rc = LaunchOp<T>(op, in + B->in_off[c], o, no ? o + no : nullptr,
                                  no ? o + 2 * no : nullptr, nullptr, nullptr,
                                  B->streams[B->stream_of[c]]);
        if (rc)
            return rc;
    }
    for (size_t k = 0; k < B->streams.size(); ++k)
    {
        NKB_CUDA_TRY(cudaEventRecord(B->joins[k], B->streams[k]));
        NKB_CUDA_TRY(cudaStreamWaitEvent(s, B->joins[k], 0));
    }
    return NKB_OK;
}
// launch the batch's graph on `run`, capturing it first when (in, out)
// changed; timed by ev0 / ev1
template <typename T> int RunGraph(nkb_batch *B, const T *din, T *dout, cudaStream_t run)
{
    // one graph per (input, output) pair; re-captured when they change
    if (!B->graph || B->g_in != din || B->g_out != dout)
    {
        if (B->graph)
            cudaGraphExecDestroy(B->graph);
        B->graph = nullptr;
        cudaStream_t cap;
        NKB_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t g;
        cudaError_t ce = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        int rc         = ce == cudaSuccess ? LaunchAll<T>(B, din, dout, cap) : NKB_OK;
        cudaError_t ee = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc)
            return rc;
        if (ce != cudaSuccess || ee != cudaSuccess)
            return SetError(NKB_ERR_CUDA, "nkb_batch_apply: capture: %s",
                            cudaGetErrorString(ce != cudaSuccess ? ce : ee));
        ce = cudaGraphInstantiate(&B->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess)
            return SetError(NKB_ERR_CUDA, "nkb_batch_apply: instantiate: %s", cudaGetErrorString(ce));
        B->g_in  = din;
        B->g_out = dout;
    }
    NKB_CUDA_TRY(cudaEventRecord(B->ev0, run));
    NKB_CUDA_TRY(cudaGraphLaunch(B->graph, run));
    NKB_CUDA_TRY(cudaEventRecord(B->ev1, run));
    return NKB_OK;
}
} // namespace

extern "C" int nkb_batch_create(nkb_op *const *ops, int nops, int nstreams, nkb_batch **out)
{
    ClearError();
    if (!ops || nops < 1 || !out)
        return SetError(NKB_ERR_INVALID, "nkb_batch_create: bad arguments");
    *out = nullptr;
    for (int c = 0; c < nops; ++c)
    {
        if (!ops[c])
            return SetError(NKB_ERR_INVALID, "nkb_batch_create: op %d is NULL", c);
        if (ops[c]->optype != ops[0]->optype || ops[c]->device != ops[0]->device ||
            ops[c]->precision != ops[0]->precision)
            return SetError(NKB_ERR_INVALID, "nkb_batch_create: all operators must be of one "
                                             "type and precision on one device");
    }
    if (nstreams <= 0)
        nstreams = 4;
    nstreams     = std::min(nstreams, nops);
    nkb_batch *B = new nkb_batch();
    B->device    = ops[0]->device;
    B->precision = ops[0]->precision;
    B->ops.assign(ops, ops + nops);
    B->nout = ops[0]->optype == NKB_PHYSDERIV ? 3 : 1;
    for (nkb_op *op : B->ops)
    {
        long ni = 0, no = 0;
        nkb_op_sizes(op, &ni, &no);
        B->in_off.push_back(B->in_size);
        B->out_off.push_back(B->out_size);
        B->in_size += ni;
        B->out_size += no * B->nout;
    }
    // largest first, each to the least-loaded stream
    B->order.resize(nops);
    std::iota(B->order.begin(), B->order.end(), 0);
    std::stable_sort(B->order.begin(), B->order.end(),
                     [&](int a, int b) { return Cost(B->ops[a]) > Cost(B->ops[b]); });
    std::vector<double> load(nstreams, 0.0);
    B->stream_of.assign(nops, 0);
    for (int c : B->order)
    {
        const int k = int(std::min_element(load.begin(), load.end()) - load.begin());
        B->stream_of[c] = k;
        load[k] += Cost(B->ops[c]);
    }
    auto fail = [&](int rc) {
        nkb_batch_destroy(B);
        return rc;
    };
    if (cudaSetDevice(B->device) != cudaSuccess)
        return fail(SetError(NKB_ERR_CUDA, "nkb_batch_create: device %d", B->device));
    B->streams.assign(nstreams, nullptr);
    B->joins.assign(nstreams, nullptr);
    for (int k = 0; k < nstreams; ++k)
        if (cudaStreamCreateWithFlags(&B->streams[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&B->joins[k], cudaEventDisableTiming) != cudaSuccess)
            return fail(SetError(NKB_ERR_CUDA, "nkb_batch_create: streams"));
    if (cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&B->order_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&B->ev0) != cudaSuccess || cudaEventCreate(&B->ev1) != cudaSuccess ||
        cudaStreamCreateWithFlags(&B->own, cudaStreamNonBlocking) != cudaSuccess)
        return fail(SetError(NKB_ERR_CUDA, "nkb_batch_create: events"));
    *out = B;
    return NKB_OK;
}

extern "C" int nkb_batch_sizes(const nkb_batch *B, long *in_size, long *out_size)
{
    if (!B)
        return SetError(NKB_ERR_INVALID, "nkb_batch_sizes: NULL batch");
    if (in_size)
        *in_size = B->in_size;
    if (out_size)
        *out_size = B->out_size;
    return NKB_OK;
}

extern "C" int nkb_batch_apply(nkb_batch *B, const double *in, double *out, int flags, void *stream)
{
    ClearError();
    if (!B || !in || !out)
        return SetError(NKB_ERR_INVALID, "nkb_batch_apply: NULL argument");
    if (B->precision != NKB_FP64)
        return SetError(NKB_ERR_INVALID, "nkb_batch_apply: FP32 batch; use nkb_batch_apply_f32");
    NKB_CUDA_TRY(cudaSetDevice(B->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool legacy = s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread;
    cudaStream_t run  = legacy ? B->own : s;
    const double *din = in;
    double *dout      = out;
    if (flags & NKB_HOST_PTRS)
    {
        if (!B->stage && cudaMalloc(&B->stage, (B->in_size + B->out_size) * sizeof(double)) !=
                             cudaSuccess)
            return SetError(NKB_ERR_NOMEM, "nkb_batch_apply: staging buffers");
        NKB_CUDA_TRY(cudaMemcpyAsync(B->stage, in, B->in_size * sizeof(double),
                                     cudaMemcpyHostToDevice, run));
        din  = B->stage;
        dout = B->stage + B->in_size;
    }
    else if (legacy)
    {
        // order the private stream after the caller's earlier work
        NKB_CUDA_TRY(cudaEventRecord(B->order_ev, s));
        NKB_CUDA_TRY(cudaStreamWaitEvent(run, B->order_ev, 0));
    }
    int rc = RunGraph<double>(B, din, dout, run);
    if (rc)
        return rc;
    if (flags & NKB_HOST_PTRS)
    {
        NKB_CUDA_TRY(cudaMemcpyAsync(out, dout, B->out_size * sizeof(double),
                                     cudaMemcpyDeviceToHost, run));
        NKB_CUDA_TRY(cudaStreamSynchronize(run));
        for (nkb_op *op : B->ops)
            if ((rc = CheckOpError(op)))
                return rc;
    }
    else if (legacy)
    {
        NKB_CUDA_TRY(cudaEventRecord(B->order_ev, run));
        NKB_CUDA_TRY(cudaStreamWaitEvent(s, B->order_ev, 0));
    }
    return NKB_OK;
}

extern "C" int nkb_batch_apply_f32(nkb_batch *B, const float *in, float *out, void *stream)
{
    ClearError();
    if (!B || !in || !out)
        return SetError(NKB_ERR_INVALID, "nkb_batch_apply_f32: NULL argument");
    if (B->precision != NKB_FP32)
        return SetError(NKB_ERR_INVALID, "nkb_batch_apply_f32: FP64 batch; use nkb_batch_apply");
    NKB_CUDA_TRY(cudaSetDevice(B->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool legacy = s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread;
    cudaStream_t run  = legacy ? B->own : s;
    if (legacy)
    {
        NKB_CUDA_TRY(cudaEventRecord(B->order_ev, s));
        NKB_CUDA_TRY(cudaStreamWaitEvent(run, B->order_ev, 0));
    }
    int rc = RunGraph<float>(B, in, out, run);
    if (rc)
        return rc;
    if (legacy)
    {
        NKB_CUDA_TRY(cudaEventRecord(B->order_ev, run));
        NKB_CUDA_TRY(cudaStreamWaitEvent(s, B->order_ev, 0));
    }
    return NKB_OK;
}

extern "C" int nkb_batch_last_ms(nkb_batch *B, float *ms)
{
    if (!B || !ms)
        return SetError(NKB_ERR_INVALID, "nkb_batch_last_ms: NULL argument");
    NKB_CUDA_TRY(cudaSetDevice(B->device));
    NKB_CUDA_TRY(cudaEventSynchronize(B->ev1));
    NKB_CUDA_TRY(cudaEventElapsedTime(ms, B->ev0, B->ev1));
    return NKB_OK;
}

extern "C" void nkb_batch_destroy(nkb_batch *B)
{
    if (!B)
        return;
    cudaSetDevice(B->device);
    for (cudaStream_t w : B->streams)
        if (w)
            cudaStreamSynchronize(w);
    if (B->own)
        cudaStreamSynchronize(B->own);
    if (B->graph)
        cudaGraphExecDestroy(B->graph);
    for (cudaStream_t w : B->streams)
        if (w)
            cudaStreamDestroy(w);
    for (cudaEvent_t e : B->joins)
        if (e)
            cudaEventDestroy(e);
    for (cudaEvent_t e : {B->fork, B->ev0, B->ev1, B->order_ev})
        if (e)
            cudaEventDestroy(e);
    if (B->own)
        cudaStreamDestroy(B->own);
    cudaFree(B->stage);
    delete B;
}
