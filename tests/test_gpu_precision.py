"""The precision forms on the GPU: the FP16 system matrix (values, scales,
its transpose, sensitivity, MLEM within 1e-3 relative L2 of an FP64
oracle) and the FP64 MLEM used as the full-size yardstick."""
import numpy as np
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu

SEED = 1251
HALF_RTOL = 1e-3      # FP16 matrix image vs FP64 oracle (relative L2)
F64_RTOL = 1e-10      # GPU FP64 iteration vs CPU FP64 oracle
F32_RTOL = 1e-4       # FP32 iteration vs GPU FP64 iteration


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


@pytest.fixture(scope="module")
def setup(rlib, torch):
    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    lst = np.arange(g.n_channels, dtype=np.int32)
    A = ctx.build(lst, 100, SEED)
    A.to_half()
    rp, col, val = A.to_numpy()
    from oracle import oracle as O

    xt = cfg.phantom(g, rods=False)
    lam = O.spmv(0, A.m, A.n, rp, col, val, xt.astype(np.float64), dtype=np.float64)
    y = cfg.poisson_measurement(lam, 2e6, seed=7)
    return ctx, A, (rp, col, val), y


def measured(rp, col, val, y):
    rows = np.nonzero(y != 0)[0]
    rp_m = np.concatenate([[0], np.cumsum(np.diff(rp)[rows])]).astype(np.int64)
    col_m = np.concatenate([col[rp[r]:rp[r + 1]] for r in rows]).astype(np.int32)
    val_m = np.concatenate([val[rp[r]:rp[r + 1]] for r in rows])
    return rows, rp_m, col_m, val_m


def test_half_values_and_scales(setup):
    ctx, A, (rp, col, val), y = setup
    h = A.hval.cpu().numpy().astype(np.float64)
    sc = A.rscale.cpu().numpy()
    rows = np.repeat(np.arange(A.m), np.diff(rp))
    # scale = row max * 2^-15 exactly
    mx = np.zeros(A.m, np.float32)
    np.maximum.at(mx, rows, np.abs(val))
    want = np.where(mx > 0, np.ldexp(mx, -15), np.float32(1)).astype(np.float32)
    assert np.array_equal(sc.view(np.uint32), want.view(np.uint32))
    assert h.max() <= 32768.0
    approx = h * sc[rows].astype(np.float64)
    normal = h >= 2.0 ** -14
    rel = np.abs(approx[normal] - val[normal]) / val[normal]
    assert rel.max() <= 2.0 ** -11 * 1.0001
    assert np.all(np.abs(approx[~normal] - val[~normal]) <= 2.0 ** -25 * sc[rows][~normal])


def test_half_transpose_matches_rows(setup):
    ctx, A, (rp, col, val), y = setup
    order = A.row_order.cpu().numpy()
    cp = A.col_ptr.cpu().numpy()
    pos = A.row_idx.cpu().numpy()
    ht = A.htval.cpu().numpy().view(np.uint16)
    hv = A.hval.cpu().numpy().view(np.uint16)
    rows = np.repeat(np.arange(A.m), np.diff(rp))
    rank = np.empty(A.m, np.int64)
    rank[order] = np.arange(A.m)
    o = np.lexsort((rank[rows], col))
    assert np.array_equal(ht, hv[o])
    assert np.array_equal(A.pscale.cpu().numpy(), A.rscale.cpu().numpy()[order])


def test_sensitivity_half_fp64(rlib, setup):
    ctx, A, (rp, col, val), y = setup
    s64, s32 = rlib.sensitivity_half(A)
    h = A.hval.cpu().numpy().astype(np.float64)
    sc = A.rscale.cpu().numpy().astype(np.float64)
    rows = np.repeat(np.arange(A.m), np.diff(rp))
    want = np.bincount(col, weights=h * sc[rows], minlength=A.n)
    assert np.allclose(s64.cpu().numpy(), want, rtol=1e-12, atol=0)
    assert abs(float(s32.double().sum()) - 1.0) < 1e-5


def test_mlem_f64_matches_cpu_fp64_oracle(rlib, oracle, torch, setup):
    ctx, A, (rp, col, val), y = setup
    rows, rp_m, col_m, val_m = measured(rp, col, val, y)
    s_all = oracle.column_sums_f64(A.m, A.n, rp, col, val)
    s = s_all / s_all.sum()
    x0 = np.full(A.n, 1.0 / A.n)
    want = oracle.mlem(rows.size, A.n, rp_m, col_m, val_m, y[rows].astype(np.float64), s, x0, 10, dtype=np.float64)
    x = torch.from_numpy(x0.copy()).cuda()
    ll = ctx.mlem_f64(A, torch.from_numpy(y).cuda(), torch.from_numpy(s).cuda(), x, 10, loglik=True)
    x = x.cpu().numpy()
    assert np.linalg.norm(x - want) / np.linalg.norm(want) < F64_RTOL
    assert np.all(np.diff(ll) >= 0)


def test_mlem_fp32_and_fp16_against_fp64(rlib, oracle, torch, setup):
    ctx, A, (rp, col, val), y = setup
    yt = torch.from_numpy(y).cuda()
    s64, s32 = rlib.sensitivity(A)
    x64 = torch.full((A.n,), 1.0 / A.n, dtype=torch.float64, device="cuda")
    ctx.mlem_f64(A, yt, s64 / s64.sum(), x64, 20)
    ref = x64.cpu().numpy()
    # FP32 matrix and vectors
    x32 = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ctx.mlem(A, yt, s32, x32, 20)
    x32 = x32.double().cpu().numpy()
    assert np.linalg.norm(x32 - ref) / np.linalg.norm(ref) < F32_RTOL
    # FP16 matrix with its own sensitivity, compensated back projection
    h64, h32 = rlib.sensitivity_half(A)
    xh = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ll = ctx.mlem_half(A, yt, h32, xh, 20, loglik=True)
    xh = xh.double().cpu().numpy()
    rel = np.linalg.norm(xh - ref) / np.linalg.norm(ref)
    assert rel < HALF_RTOL, rel
    assert abs(xh.sum() - 1.0) < 1e-5
    assert np.all(np.diff(ll) >= -1e-6 * abs(ll[-1]))
    # graph and non-graph launches agree
    xg = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ctx.mlem_half(A, yt, h32, xg, 20, use_graph=True)
    xn = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ctx.mlem_half(A, yt, h32, xn, 20, use_graph=False)
    assert torch.equal(xg, xn)


def test_half_needs_transpose_first(rlib, torch):
    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    A = ctx.build(np.arange(100, dtype=np.int32), 10, SEED)
    assert rlib.lib().raptr_matrix_half(A._h, None) != 0  # RAPTR_ERR_INVALID, no fault
    with pytest.raises(RuntimeError):
        rlib.sensitivity_half(A)
