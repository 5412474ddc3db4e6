"""Row-sharded MLEM across ranks (one GPU per rank).

The channel rows of the system matrix are split into contiguous shards, one
per rank, as the reference splits its channel chunks over MPI ranks
(src/tests/reco.cu:237-275).  Each rank builds and keeps its own rows; per
iteration it forward-projects its rows, back-projects them into a partial
correction image, and the partial images are summed over all ranks (the
reference's MPI_Allreduce, src/tests/reco.cu:279-281; here NCCL over NVLink).
The update x*c/(s+(s==0)) and the normalisation are then identical on every
rank.  The sensitivity is summed the same way, in FP64.

The compute is supplied by an `ops` object (the GPU implementation is
`GpuShardOps`), the reduction by a torch.distributed-like `comm`.
"""
from __future__ import annotations

from typing import Tuple


def shard_bounds(n_rows: int, world: int, rank: int) -> Tuple[int, int]:
    """Rows [lo, hi) of `rank` when n_rows are split into `world` contiguous
    shards whose sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    return rank * n_rows // world, (rank + 1) * n_rows // world


class GpuShardOps:
    """The four MLEM pieces on one rank's rows, through the C ABI.  The
    matrix must carry its transpose (Matrix.transpose())."""

    def __init__(self, A):
        import torch

        import raptr_b200 as R

        if not A.has_transpose:
            A.transpose()
        self.R, self.A = R, A
        self.e = torch.empty(A.m, device=A.row_ptr.device)
        self.c = torch.empty(A.n, device=A.row_ptr.device)
        self.acc = torch.zeros(1, dtype=torch.float64, device=A.row_ptr.device)

    def column_sums(self):
        s64, _ = self.R.sensitivity(self.A)
        return s64

    def forward(self, y, x):
        self.R.mlem_forward(self.A, y, x, self.e)
        return self.e

    def back(self, e):
        self.R.mlem_back(self.A, e, self.c)
        return self.c

    def update(self, x, c, s):
        self.R.mlem_update(x, c, s, self.acc)


class ShardedMLEM:
    def __init__(self, ops, comm):
        self.ops = ops
        self.comm = comm

    def sensitivity(self):
        """Normalised sensitivity: FP64 column sums of all ranks' rows."""
        s64 = self.ops.column_sums()
        if self.comm is not None:
            self.comm.all_reduce(s64)
        return (s64 / s64.sum()).float()

    def iterate(self, y, s, x, n_iter: int):
        for _ in range(n_iter):
            e = self.ops.forward(y, x)
            c = self.ops.back(e)
            if self.comm is not None:
                self.comm.all_reduce(c)
            self.ops.update(x, c, s)
        return x
