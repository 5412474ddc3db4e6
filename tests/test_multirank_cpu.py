"""Row-sharded MLEM across ranks (raptr_b200.distributed) on CPU: two gloo
ranks, each with its own contiguous block of rows, must reproduce the
single-rank reconstruction.  The per-rank compute here is CPU restatement
(oracle SpMVs); the decomposition, the all-reduces and the update order are
the ones bench.py runs on GPUs with NCCL."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from raptr_b200 import config as cfg
from raptr_b200.distributed import ShardedMLEM, shard_bounds


class OracleShardOps:
    """CPU stand-in for GpuShardOps on one shard of rows."""

    def __init__(self, O, rp, col, val, n):
        self.O, self.rp, self.col, self.val, self.n = O, rp, col, val, n
        self.m = rp.size - 1

    def column_sums(self):
        return torch.from_numpy(self.O.column_sums_f64(self.m, self.n, self.rp, self.col, self.val))

    def forward(self, y, x):
        yt = self.O.spmv(0, self.m, self.n, self.rp, self.col, self.val, x.numpy())
        yn = y.numpy()
        e = np.where(yn != 0, yn / np.where(yt == 0, 1, yt), 0).astype(np.float32)
        return torch.from_numpy(e)

    def back(self, e):
        return torch.from_numpy(self.O.spmv(1, self.m, self.n, self.rp, self.col, self.val, e.numpy()))

    def update(self, x, c, s):
        sn = s.numpy()
        dvs = sn + (sn == 0)
        xx = (x.numpy() * c.numpy() / dvs).astype(np.float32)
        scale = np.float32(1.0 / np.float32(xx.astype(np.float64).sum()))
        x.copy_(torch.from_numpy((scale * xx).astype(np.float32)))


def problem():
    from oracle import oracle as O

    g = cfg.SMALL
    lst = np.arange(0, g.n_channels, 53, dtype=np.int32)
    rp, col, val = O.sysmat(g, lst, 20, 1251, method=1)
    xt = cfg.phantom(g, rods=False)
    y = (O.spmv(0, lst.size, g.n_voxels, rp, col, val, xt) * 1e4).astype(np.float32)
    y[::7] = 0  # some unmeasured channels
    return O, g, rp, col, val, y


def rows_of(rp, col, val, lo, hi):
    b, e = rp[lo], rp[hi]
    return (rp[lo:hi + 1] - b).astype(np.int64), col[b:e].copy(), val[b:e].copy()


def rank_main(rank, world, port, out, n_iter):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        O, g, rp, col, val, y = problem()
        m = rp.size - 1
        lo, hi = shard_bounds(m, world, rank)
        ops = OracleShardOps(O, *rows_of(rp, col, val, lo, hi), g.n_voxels)
        mlem = ShardedMLEM(ops, dist)
        s = mlem.sensitivity()
        x = torch.full((g.n_voxels,), np.float32(1.0 / g.n_voxels))
        mlem.iterate(torch.from_numpy(y[lo:hi]), s, x, n_iter)
        if rank == 0:
            np.save(out, x.numpy())
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_bounds_cover_rows_once():
    for n in (0, 1, 7, 1000, 5140980):
        for w in (1, 2, 3, 8):
            b = [shard_bounds(n, w, r) for r in range(w)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))
            assert max(h - l for l, h in b) - min(h - l for l, h in b) <= 1
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks_reproduce_single_rank(tmp_path, world):
    out = str(tmp_path / "x.npy")
    mp.start_processes(rank_main, args=(world, free_port(), out, 5), nprocs=world, start_method="spawn", join=True)
    xs = np.load(out)
    O, g, rp, col, val, y = problem()
    ops = OracleShardOps(O, rp, col, val, g.n_voxels)
    single = ShardedMLEM(ops, None)
    s = single.sensitivity()
    x = torch.full((g.n_voxels,), np.float32(1.0 / g.n_voxels))
    single.iterate(torch.from_numpy(y), s, x, 5)
    x = x.numpy()
    assert np.linalg.norm(xs - x) / np.linalg.norm(x) < 1e-5
    # and the sharded result is MLEM of the measured rows (oracle loop)
    meas = np.nonzero(y)[0]
    rpm = np.concatenate([[0], np.cumsum(np.diff(rp)[meas])]).astype(np.int64)
    colm = np.concatenate([col[rp[r]:rp[r + 1]] for r in meas])
    valm = np.concatenate([val[rp[r]:rp[r + 1]] for r in meas])
    want = O.mlem(meas.size, g.n_voxels, rpm, colm, valm, y[meas], s.numpy(),
                  np.full(g.n_voxels, np.float32(1.0 / g.n_voxels), np.float32), 5)
    assert np.linalg.norm(xs - want) / np.linalg.norm(want) < 1e-4
