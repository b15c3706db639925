"""Batched application of every collection of a mixed-element mesh in one
call (concurrent streams, one CUDA graph): the same bits as applying the
collections one by one, for each operator type, through host and device
pointers."""
import numpy as np
import pytest

import nektar_b200 as nb
from nektar_b200.mixed_mesh import MixedMesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("optype", ["helmholtz", "linear_adr", "bwdtrans", "iproduct",
                                    "iproduct_deriv", "physderiv"])
def test_batch_equals_collection_by_collection(optype):
    mm = MixedMesh(n=6, ncells=(60, 50, 40), pmin=2, pmax=5, seed=2)
    cols = mm.collections(optype, lam=2.5)
    ops = [op for _, op in cols]
    B = nb.Batch(ops, nstreams=3)
    x = np.random.default_rng(0).uniform(-1, 1, B.in_size)
    y = B(x)
    parts, o = [], 0
    for op in ops:
        xi = x[o:o + op.in_size]
        o += op.in_size
        r = op(xi)
        parts.extend(r if isinstance(r, (tuple, list)) else [r])
    ref = np.concatenate([np.ravel(p) for p in parts])
    assert y.size == ref.size == B.out_size
    assert np.array_equal(y, ref)
    # a second call reuses the captured graph
    assert np.array_equal(B(x), ref)
    B.close()


def test_batch_device_pointers_and_regraph():
    import torch
    mm = MixedMesh(n=5, ncells=(30, 30, 20), pmin=3, pmax=4, seed=5)
    ops = [op for _, op in mm.collections("helmholtz")]
    B = nb.Batch(ops)
    x = np.random.default_rng(1).uniform(-1, 1, B.in_size)
    ref = B(x)
    xd = torch.from_numpy(x).cuda()
    for _ in range(2):  # new output buffer each time: the graph is re-captured
        yd = torch.empty(B.out_size, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        B.apply_device(xd.data_ptr(), yd.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(yd.cpu().numpy(), ref)
    assert B.last_ms() > 0
    B.close()


@pytest.mark.parametrize("optype", ["helmholtz", "linear_adr", "iproduct_deriv"])
def test_fp32_batch_equals_collection_by_collection(optype):
    """FP32 operators in one batch (the FP32 variant of the mixed-element
    launch): the same bits as each collection applied alone."""
    import torch
    mm = MixedMesh(n=6, ncells=(60, 50, 40), pmin=2, pmax=6, seed=3)
    ops = []
    for m in mm.meshes():
        op = nb.Operator(optype, m, precision="fp32")
        if optype != "iproduct_deriv":
            op.set_factors(1.5)
        ops.append(op)
    B = nb.Batch(ops, nstreams=3)
    x = torch.rand(B.in_size, dtype=torch.float32, device="cuda") * 2 - 1
    y = torch.empty(B.out_size, dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    B.apply_device(x.data_ptr(), y.data_ptr(), stream=s)
    ref = torch.empty_like(y)
    oi = oo = 0
    for op in ops:
        op.apply_device(x[oi:].data_ptr(), ref[oo:].data_ptr(), stream=s)
        oi += op.in_size
        oo += op.out_size
    torch.cuda.synchronize()
    assert torch.equal(y, ref)
    with pytest.raises(nb.NektarB200Error):
        B(np.zeros(B.in_size))  # host FP64 entry point refuses an FP32 batch
    B.close()
