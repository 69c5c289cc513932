"""One process per GPU running independent solves (replicas).

The solve is not sharded across GPUs (one B200 per solve), so the only
coordination between ranks is timing: a barrier around the timed region, the
maximum of the ranks' times, and the sum of the solves they completed.  The
helpers work on any torch.distributed backend (NCCL on GPUs, gloo on CPU for
the tests) and keep every rank on the same sequence of collectives.
"""
from __future__ import annotations

import datetime
import os


def world():
    return (int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=600):
    """Initialises the process group when WORLD_SIZE > 1; returns
    (world_size, rank, local_rank)."""
    import torch
    import torch.distributed as dist
    ws, rank, local = world()
    if ws > 1 and not dist.is_initialized():
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend,
                                timeout=datetime.timedelta(seconds=timeout_s),
                                **kw)
    elif ws == 1 and backend == "nccl" and torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def _device():
    import torch
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier():
    """Barrier across ranks, then a device synchronise when on a GPU."""
    import torch
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()


def _reduce(value, op):
    import torch
    import torch.distributed as dist
    if not (dist.is_initialized() and dist.get_world_size() > 1):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=op)
    return t.item()


def max_over_ranks(value):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX)


def sum_over_ranks(value):
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM)


def throughput(units_done, seconds):
    """Whole-job rate: units of all ranks over the slowest rank's time."""
    return sum_over_ranks(units_done) / max_over_ranks(seconds)


def rhs_seed(rank, base=1000):
    """Every replica draws its own right-hand sides."""
    return base + rank


def shutdown():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()
