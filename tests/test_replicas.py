"""Replica bookkeeping of runs on several GPUs, on the CPU with two gloo
ranks: every rank gets the slowest rank's time, and whole-job throughput
counts every rank's units over that time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from nektar_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    pg = replicas.init(world, rank, backend="gloo", timeout_s=60)
    ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
    ms_max = replicas.max_over_ranks(ms, pg)
    rate = replicas.whole_job_rate(4, world, ms_max)
    replicas.barrier(pg)
    out[rank] = (ms_max, rate)
    replicas.finish(pg)


def test_max_over_ranks_and_whole_job_rate_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1]
        ms_max, rate = out[0]
        assert ms_max == 150.0
        assert rate == pytest.approx(2 * 4 / 0.150)


def test_single_process_needs_no_group():
    assert replicas.init(1, 0) is None
    assert replicas.max_over_ranks(3.5, None) == 3.5
    assert replicas.whole_job_rate(2, 1, 500.0) == pytest.approx(4.0)
