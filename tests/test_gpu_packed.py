"""The delta-coded FP16 form: raptr_pack_half's runs decode to the FP16
matrix's entries (steps above 65535 included), and MLEM over them gives the
FP16 iteration's image and stays within 1e-3 relative L2 of FP64."""
from types import SimpleNamespace

import numpy as np
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu

SEED = 1251
HALF_RTOL = 1e-3    # FP16 matrix image vs FP64 iteration (relative L2)
SAME_RTOL = 1e-5    # delta-coded vs plain FP16 iteration (summation order only)


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def decode(seg, anchor, words):
    """Run, index and binary16 bits of every word of the runs."""
    seg = np.asarray(seg, np.int64)
    w = np.asarray(words).view(np.uint32)
    assert w.size == 4 * seg[-1]
    count = seg.size - 1
    runs = np.repeat(np.arange(count), 4 * np.diff(seg))
    cs = np.concatenate([[0], np.cumsum((w & 0xFFFF).astype(np.int64))])
    idx = np.asarray(anchor, np.int64)[runs] + cs[1:] - cs[4 * seg[:-1]][runs]
    return runs, idx, (w >> 16).astype(np.uint16)


def check_runs(seg, anchor, words, ptr, idx, hv, n):
    """The decoded runs hold the entries of (ptr, idx, hv) in order; the
    other words (steps above 65535, padding) carry value 0 and indices
    inside the run's range."""
    runs, di, dh = decode(seg, anchor, words)
    assert di.min(initial=0) >= 0 and di.max(initial=0) < max(n, 1)
    ptr, idx, hv = (np.asarray(a) for a in (ptr, idx, hv))
    rows = np.repeat(np.arange(ptr.size - 1), np.diff(ptr))
    keep = hv.view(np.uint16) != 0
    dk = dh != 0
    np.testing.assert_array_equal(runs[dk], rows[keep])
    np.testing.assert_array_equal(di[dk], idx[keep])
    np.testing.assert_array_equal(dh[dk], hv.view(np.uint16)[keep])
    # every run covers exactly its entries' indices, ascending
    for r in np.unique(rows)[:200]:
        sel = runs == r
        assert np.all(np.diff(di[sel]) >= 0)
        assert di[sel][0] == idx[ptr[r]]
    # words beyond the entries: the steps above 65535 and at most 3 of
    # padding per run
    first = np.r_[True, rows[1:] != rows[:-1]] if rows.size else np.zeros(0, bool)
    steps = np.where(first, 0, np.diff(idx.astype(np.int64), prepend=0))
    escapes = int(np.sum(np.where(steps > 65535, (steps - 1) // 65535, 0)))
    assert idx.size + escapes <= words.size <= idx.size + escapes + 3 * (ptr.size - 1)


@pytest.fixture(scope="module")
def small(rlib, torch):
    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    A = ctx.build(np.arange(g.n_channels, dtype=np.int32), 100, SEED)
    A.to_packed()
    from oracle import oracle as O

    rp, col, val = A.to_numpy()
    lam = O.spmv(0, A.m, A.n, rp, col, val, cfg.phantom(g, rods=False).astype(np.float64), dtype=np.float64)
    y = cfg.poisson_measurement(lam, 2e6, seed=7)
    return ctx, A, y


def test_packed_runs_decode_to_the_fp16_matrix(rlib, torch, small):
    _, A, _ = small
    check_runs(A.pseg.cpu().numpy(), A.panchor.cpu().numpy(), A.pword.cpu().numpy(), A.row_ptr.cpu().numpy(),
               A.col.cpu().numpy(), A.hval.cpu().numpy(), A.n)
    check_runs(A.tseg.cpu().numpy(), A.tanchor.cpu().numpy(), A.tword.cpu().numpy(), A.col_ptr.cpu().numpy(),
               A.row_idx.cpu().numpy(), A.htval.cpu().numpy(), A.m)
    # 4 bytes per entry and a little padding, against 6 for the plain FP16 form
    assert A.pword.numel() < 1.02 * A.nnz + 4 * A.m


def test_packed_mlem_equals_fp16_and_fp64(rlib, torch, small):
    ctx, A, y = small
    yt = torch.from_numpy(y).cuda()
    s64, _ = rlib.sensitivity(A)
    x64 = torch.full((A.n,), 1.0 / A.n, dtype=torch.float64, device="cuda")
    ctx.mlem_f64(A, yt, s64 / s64.sum(), x64, 20)
    ref = x64.cpu().numpy()
    _, h32 = rlib.sensitivity_half(A)
    xh = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ctx.mlem_half(A, yt, h32, xh, 20)
    xp = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ll = ctx.mlem_packed(A, yt, h32, xp, 20, loglik=True)
    xh, xpn = xh.double().cpu().numpy(), xp.double().cpu().numpy()
    assert np.linalg.norm(xpn - xh) / np.linalg.norm(xh) < SAME_RTOL
    assert np.linalg.norm(xpn - ref) / np.linalg.norm(ref) < HALF_RTOL
    assert abs(xpn.sum() - 1.0) < 1e-5
    assert np.all(np.diff(ll) >= -1e-6 * abs(ll[-1]))
    # graph and stream launches agree
    xg = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ctx.mlem_packed(A, yt, h32, xg, 20, use_graph=False)
    assert torch.equal(xg, xp)


def synthetic(torch, m, n, seed):
    """A CSR with wide column gaps (many steps above 65535, empty rows) and
    binary16 values, its transpose in natural row order."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 40, m)
    lens[::17] = 0
    cols = [np.sort(rng.choice(n, size=k, replace=False)) for k in lens]
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    col = np.concatenate(cols).astype(np.int32)
    hv = rng.uniform(0.01, 2.0, col.size).astype(np.float16)
    import raptr_b200 as R

    rp_t, col_t = torch.from_numpy(rp).cuda(), torch.from_numpy(col).cuda()
    cp, ri, tv = R.csr_transpose(m, n, rp_t, col_t, torch.from_numpy(hv.astype(np.float32)).cuda())
    return rp_t, col_t, torch.from_numpy(hv.view(np.int16)).cuda(), cp, ri, tv.half().view(torch.int16)


def test_pack_steps_above_65535(rlib, torch):
    m, n = 3000, 3_000_000
    rp, col, hv, cp, ri, htv = synthetic(torch, m, n, 5)
    seg, anc, words = rlib.pack_half(rp, col, hv)
    assert int(np.sum(np.diff(col.cpu().numpy().astype(np.int64)) > 65535)) > 100
    check_runs(seg.cpu().numpy(), anc.cpu().numpy(), words.cpu().numpy(), rp.cpu().numpy(), col.cpu().numpy(),
               hv.cpu().numpy(), n)
    tseg, tanc, twords = rlib.pack_half(cp, ri, htv)
    check_runs(tseg.cpu().numpy(), tanc.cpu().numpy(), twords.cpu().numpy(), cp.cpu().numpy(), ri.cpu().numpy(),
               htv.cpu().numpy(), m)


def test_packed_mlem_with_wide_steps_equals_fp16(rlib, torch):
    m, n = 4000, 400_000
    rp, col, hv, cp, ri, htv = synthetic(torch, m, n, 9)
    ctx = rlib.Context(cfg.SMALL, 0)
    ones = torch.ones(m, device="cuda")
    A = SimpleNamespace(m=m, n=n, row_ptr=rp, col=col, hval=hv, rscale=ones, col_ptr=cp, row_idx=ri, htval=htv,
                        row_rank=None)
    P = SimpleNamespace(m=m, n=n, rscale=ones, row_rank=None)
    P.pseg, P.panchor, P.pword = rlib.pack_half(rp, col, hv)
    P.tseg, P.tanchor, P.tword = rlib.pack_half(cp, ri, htv)
    y = torch.from_numpy(np.random.default_rng(3).poisson(5.0, m).astype(np.float32)).cuda()
    s = torch.zeros(n, device="cuda").index_add_(0, col.long(), hv.view(torch.float16).float())
    s = s / s.sum()
    xh = torch.full((n,), np.float32(1.0 / n), device="cuda")
    ctx.mlem_half(A, y, s, xh, 8)
    xp = torch.full((n,), np.float32(1.0 / n), device="cuda")
    ctx.mlem_packed(P, y, s, xp, 8)
    assert float(torch.linalg.norm(xp - xh) / torch.linalg.norm(xh)) < SAME_RTOL


def test_pack_rejects_bad_input(rlib, torch):
    rp = torch.tensor([0, 3], dtype=torch.int64, device="cuda")
    col = torch.tensor([5, 2, 9], dtype=torch.int32, device="cuda")  # descends
    hv = torch.ones(3, dtype=torch.int16, device="cuda")
    with pytest.raises(RuntimeError):
        rlib.pack_half(rp, col, hv)
    col = torch.tensor([2, 5, 9], dtype=torch.int32, device="cuda")
    seg = torch.empty(2, dtype=torch.int64, device="cuda")
    anc = torch.empty(1, dtype=torch.int32, device="cuda")
    words = torch.empty(4, dtype=torch.int32, device="cuda")
    import ctypes as C

    nw = C.c_int64()
    L = rlib.lib()
    assert L.raptr_pack_half(1, rp.data_ptr(), col.data_ptr(), hv.data_ptr(), seg.data_ptr(), anc.data_ptr(),
                             words.data_ptr(), 2, C.byref(nw), None) != 0  # words_cap below the 4 needed
    assert nw.value == 4
