"""A small, self-contained case of the hot kernels for `ncu` captures.

    python -m raptr_b200.profile_case [--rows R] [--offset O] [--workload full] [--build-only] [--forms]

Builds rows [O, O+R) of the workload's system matrix (the channels in id
order: 28,561 per angle at 70^3 x 180 angles, so O = 628342 starts at the
23rd angle, 46 degrees), transposes it (radix sort in the channels'
back-projection order) and runs three MLEM iterations, so that each hot
kernel (sm_dense_kernel, rs_scatter, mlem_forward_kernel,
mlem_back_kernel) launches a few times on a matrix larger than L2 but only
a few GB on the device.  --build-only stops after the build.  With --forms
it also runs the FP16 form (three iterations) and the batched form (16
frames, two iterations).

    python -m raptr_b200.profile_case --columns X0:X1 [--rows R]

The column-slab case for the back projection: every channel's row (built R
rows at a time) restricted to the voxels of x slabs [X0, X1), so that the
columns keep their full length (~10^4 entries at the centre of the 70^3
grid; the row case's columns hold a few hundred), transposed in the
library's back-projection order of the channels, then three FP32 MLEM
iterations.
"""
from __future__ import annotations

import argparse

import numpy as np


def channel_order(torch, g, m):
    """The library's back-projection order of channels 0..m-1: sorted by
    (angle, z0+z1, y0+y1, z0-z1, y0-y1), as raptr_matrix_transpose orders
    the rows of a matrix it built.  Returns (order, rank)."""
    c = torch.arange(m, dtype=torch.int64, device="cuda")
    id1y = c % g.n1y
    c = c // g.n1y
    id1z = c % g.n1z
    c = c // g.n1z
    id0y = c % g.n0y
    c = c // g.n0y
    id0z = c % g.n0z
    ida = c // g.n0z
    sz, sy = g.n0z + g.n1z - 1, g.n0y + g.n1y - 1
    k = ida
    k = k * sz + (id0z + id1z)
    k = k * sy + (id0y + id1y)
    k = k * sz + (id0z - id1z + g.n1z - 1)
    k = k * sy + (id0y - id1y + g.n1y - 1)
    order = torch.argsort(k).to(torch.int32)
    rank = torch.empty(m, dtype=torch.int32, device="cuda")
    rank[order.long()] = torch.arange(m, dtype=torch.int32, device="cuda")
    return order, rank


class _Arrays:
    """CSR + CSC arrays in the attribute layout Context.mlem reads."""
    has_transpose = True


def column_slab_case(R, torch, ctx, g, w, x0, x1, chunk):
    nyz = g.grid_n[1] * g.grid_n[2]
    c0, c1 = x0 * nyz, x1 * nyz
    M = g.n_channels
    counts, cols, vals = [], [], []
    for r0 in range(0, M, chunk):
        lst = torch.arange(r0, min(r0 + chunk, M), dtype=torch.int32, device="cuda")
        A = ctx.build(lst, w["nrays"], 1251)
        keep = (A.col >= c0) & (A.col < c1)
        pre = torch.zeros(A.nnz + 1, dtype=torch.int64, device="cuda")
        torch.cumsum(keep, 0, out=pre[1:])
        counts.append(pre[A.row_ptr[1:]] - pre[A.row_ptr[:-1]])
        cols.append((A.col[keep] - c0).to(torch.int32))
        vals.append(A.val[keep])
        del A, keep, pre
    R.trim_memory(0)  # the chunks' parked blocks: hold only the case itself on the device
    S = _Arrays()
    S.m, S.n = M, c1 - c0
    S.row_ptr = torch.zeros(M + 1, dtype=torch.int64, device="cuda")
    torch.cumsum(torch.cat(counts), 0, out=S.row_ptr[1:])
    S.col, S.val = torch.cat(cols), torch.cat(vals)
    del counts, cols, vals
    S.nnz = S.col.numel()
    order, S.row_rank = channel_order(torch, g, M)
    S.col_ptr, S.row_idx, S.tval = R.csr_transpose_ordered(S.m, S.n, S.row_ptr, S.col, S.val, order)
    del order
    torch.cuda.empty_cache()
    xt = torch.from_numpy(cfg_phantom_slab(g, w, x0, x1)).cuda()
    y = R.spmv(R.OP_N, S.m, S.n, S.row_ptr, S.col, S.val, xt) * 1000.0
    s = torch.zeros(S.n, dtype=torch.float32, device="cuda").index_add_(0, S.col.long(), S.val)
    s = s / s.sum()
    x = torch.full((S.n,), np.float32(1.0 / S.n), device="cuda")
    ctx.mlem(S, y, s, x, 3, use_graph=False)
    torch.cuda.synchronize()
    lens = (S.col_ptr[1:] - S.col_ptr[:-1]).double()
    print(f"column-slab case: x slabs [{x0}, {x1}), {S.n} columns (mean {float(lens.mean()):.0f}, max "
          f"{int(lens.max())} entries), {S.nnz} entries ({S.nnz * 8 / 1e9:.2f} GB CSR), x sum {float(x.sum()):.6f}")


def cfg_phantom_slab(g, w, x0, x1):
    from raptr_b200 import config as cfg

    return cfg.phantom(g, w["rods"]).reshape(g.grid_n[0], -1)[x0:x1].reshape(-1)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--rows", type=int, default=65536)
    p.add_argument("--offset", type=int, default=0)
    p.add_argument("--build-only", action="store_true")
    p.add_argument("--workload", default="full")
    p.add_argument("--forms", action="store_true")
    p.add_argument("--columns", default=None, help="X0:X1, the column-slab case")
    a = p.parse_args()
    import torch

    import raptr_b200 as R
    from raptr_b200 import config as cfg

    w = cfg.WORKLOADS[a.workload]
    g = w["geom"]
    ctx = R.Context(g, 0)
    if a.columns:
        x0, x1 = (int(v) for v in a.columns.split(":"))
        column_slab_case(R, torch, ctx, g, w, x0, x1, a.rows)
        return
    lst = torch.arange(a.offset, a.offset + a.rows, dtype=torch.int32, device="cuda")
    A = ctx.build(lst, w["nrays"], 1251)
    if a.build_only:
        torch.cuda.synchronize()
        print(f"profile case: {A.m} rows from {a.offset}, {A.nnz} entries (build only)")
        return
    A.transpose()
    xt = torch.from_numpy(cfg.phantom(g, w["rods"])).cuda()
    y = R.spmv(R.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, xt) * 1000.0
    s64, s = R.sensitivity(A)
    x = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ctx.mlem(A, y, s, x, 3, use_graph=False)
    if a.forms:
        A.to_half()
        h64, h = R.sensitivity_half(A)
        xh = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
        ctx.mlem_half(A, y, h, xh, 3, use_graph=False)
        K = 16
        Y = y.unsqueeze(1).repeat(1, K).contiguous()
        X = torch.full((A.n, K), np.float32(1.0 / A.n), device="cuda")
        ctx.mlem_batch(A, Y, h, X, 2, frame_tile=16, use_graph=False)
    torch.cuda.synchronize()
    print(f"profile case: {A.m} rows, {A.nnz} entries ({A.nnz * 8 / 1e9:.2f} GB CSR), x sum {float(x.sum()):.6f}")


if __name__ == "__main__":
    main()
