"""Shot sharding across ranks (one process per GPU).

Shots are independent: each rank advances its own contiguous block of shots
in its own context (bbw_set_shots), with no data-path collective.  The one
exchange is the end of the adjoint: every rank's dL/dc2q (FP64, summed over
its shots) is summed over ranks with a single all-reduce.
"""
import numpy as np


def shot_range(n_shots, rank, world):
    """Contiguous, balanced [lo, hi) block of shots for `rank`."""
    if world < 1 or not 0 <= rank < world or n_shots < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(n_shots, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def allreduce_gradient(grad, group=None, device=None):
    """Sum an FP64 gradient over the ranks of `group` (torch.distributed:
    NCCL with device tensors, gloo with host tensors); returns numpy."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(grad, np.float64))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()
