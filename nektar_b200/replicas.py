"""Replica bookkeeping for runs on several GPUs of one node.

The element operators have no exchange and one solve fits one GPU, so a run
on N GPUs is N replicas: every rank (one process per GPU, launched by
torchrun) solves its own copy. Whole-job throughput is the units all ranks
processed divided by the slowest rank's device time.
"""
import datetime


def init(world, local, backend="nccl", timeout_s=300):
    """Process group for world > 1 (None for a single process)."""
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, **kw)
    return dist


def max_over_ranks(value, pg, device="cpu"):
    """The largest of every rank's `value` (every rank gets it)."""
    if pg is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, ms_max):
    """Units per second over all ranks, timed by the slowest rank."""
    return world * units_per_rank / (ms_max / 1e3)


def barrier(pg):
    if pg is not None:
        pg.barrier()


def finish(pg):
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
