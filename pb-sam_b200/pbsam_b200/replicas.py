"""Multi-GPU plumbing: one process per GPU, independent systems per rank.

The solve has no exchange step between independent systems (poses, BD
trajectories), so ranks never communicate on the data path: each rank owns a
disjoint block of systems.  torch.distributed is used only for the barrier and
the max-over-ranks of the device time around the timed region, and for the
optional final gather of per-system results to rank 0.
"""
import os

import numpy as np


def rank_env():
    """(rank, world_size, local_rank) from the torchrun environment (defaults: single process)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_items, rank, world):
    """Contiguous block [lo, hi) of n_items owned by rank (sizes differ by at most one)."""
    if world <= 0 or rank < 0 or rank >= world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def weak_seeds(base_seed, rank):
    """Per-rank seed for weak scaling: every rank solves its own batch of systems."""
    return int(base_seed) * 1000003 + int(rank)


def max_over_ranks(value, dist=None):
    """Max of a float over all ranks (the timing reduction); identity without a process group."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None):
    """Sum of a count over all ranks (units processed by the whole job); identity without a process group."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_rows(local, dist=None):
    """Concatenate per-rank row blocks on every rank (results, not a data-path exchange)."""
    local = np.ascontiguousarray(local, dtype=np.float64)
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return local
    import torch
    world = dist.get_world_size()
    n = torch.tensor([local.shape[0]], dtype=torch.int64)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, n)
    mx = int(max(s.item() for s in sizes))
    pad = np.zeros((mx,) + local.shape[1:])
    pad[:local.shape[0]] = local
    t = torch.from_numpy(pad)
    bufs = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(bufs, t)
    return np.concatenate([b.numpy()[:int(s.item())] for b, s in zip(bufs, sizes)], axis=0)
