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
"""
from __future__ import annotations

import argparse

import numpy as np


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--rows", type=int, default=65536)
    p.add_argument("--offset", type=int, default=0)
    p.add_argument("--build-only", action="store_true")
    p.add_argument("--workload", default="full")
    p.add_argument("--forms", action="store_true")
    a = p.parse_args()
    import torch

    import raptr_b200 as R
    from raptr_b200 import config as cfg

    w = cfg.WORKLOADS[a.workload]
    g = w["geom"]
    ctx = R.Context(g, 0)
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
