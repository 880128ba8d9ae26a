"""World-size-2 gloo run of the multi-rank plumbing (CPU only)."""
import os
import socket

import numpy as np
import pytest

from pbsam_b200 import replicas


def test_shard_covers_everything_once():
    for n in (0, 1, 5, 26, 1024):
        for w in (1, 2, 3, 8):
            blocks = [replicas.shard(n, r, w) for r in range(w)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            for (a, b), (c, d) in zip(blocks, blocks[1:]):
                assert b == c and b >= a
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    r, w, _ = replicas.rank_env()
    lo, hi = replicas.shard(7, r, w)
    rows = np.arange(lo, hi, dtype=np.float64)[:, None] * np.ones((1, 3))
    allrows = replicas.gather_rows(rows, dist)
    t = replicas.max_over_ranks(1.0 + r, dist)
    u = replicas.sum_over_ranks(10.0 + r, dist)
    dist.barrier()
    if r == 0:
        np.save(out, np.concatenate([allrows.ravel(), [u, t]]))
    dist.destroy_process_group()


def test_two_rank_gather_max_and_sum(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "res.npy")
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    res = np.load(out)
    rows, u, t = res[:-2].reshape(-1, 3), res[-2], res[-1]
    assert np.array_equal(rows[:, 0], np.arange(7))
    assert t == 2.0 and u == 21.0
