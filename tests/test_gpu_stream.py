"""MLEM with rows rebuilt in every iteration (raptr_mlem_stream), the
single-GPU form of the reference's chunked reconstruction
(src/tests/reco.cu:226-275): whatever part of the matrix stays resident,
the image equals the one of the resident matrix (same scatter iteration) to
1e-5 relative L2, the computed sensitivity equals the resident matrix's,
and the image also matches the CPU oracle."""
import numpy as np
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu

SEED = 1251
NITER = 8
RTOL = 1e-5


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


@pytest.fixture(scope="module")
def case(rlib, torch):
    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    lst = np.arange(g.n_channels, dtype=np.int32)
    A = ctx.build(lst, 100, SEED)
    xt = torch.from_numpy(cfg.phantom(g, rods=False)).cuda()
    lam = rlib.spmv(rlib.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, xt).cpu().numpy()
    y = torch.from_numpy(cfg.poisson_measurement(lam, 2e6, seed=7)).cuda()
    s64, s = rlib.sensitivity(A)
    x_ref = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ctx.mlem(A, y, s, x_ref, NITER, use_graph=False)  # resident rows, scatter back projection
    return ctx, lst, A, y, s, x_ref


def rel(a, b):
    return float((a.double() - b.double()).norm() / b.double().norm())


@pytest.mark.parametrize("fraction", [0.0, 0.25, 2.0])
def test_stream_equals_resident(rlib, torch, case, fraction):
    ctx, lst, A, y, s, x_ref = case
    matrix_bytes = A.nnz * 8 + (A.m + 1) * 8
    x = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    st = ctx.mlem_stream(lst, 100, SEED, y, s, x, NITER, int(fraction * matrix_bytes))
    assert rel(x, x_ref) < RTOL
    assert st["resident_rows"] + st["streamed_rows"] == A.m
    if fraction == 0.0:
        assert st["resident_rows"] == 0 and st["resident_entries"] == 0
    elif fraction < 1.0:
        assert 0 < st["resident_rows"] < A.m
        assert st["resident_entries"] * 8 + (A.m + 1) * 8 <= fraction * matrix_bytes
        # a prefix of the rows: their entries are those of the built matrix
        assert st["resident_entries"] == int(A.row_ptr[st["resident_rows"]])
    else:
        assert st["resident_rows"] == A.m and st["resident_entries"] == A.nnz
    assert st["first_iter_ms"] > 0 and st["iter_ms"] > 0


def test_stream_computes_the_sensitivity(rlib, torch, case):
    ctx, lst, A, y, s, x_ref = case
    x = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    s_out = torch.empty(A.n, dtype=torch.float32, device="cuda")
    ctx.mlem_stream(lst, 100, SEED, y, None, x, NITER, 0, s_out=s_out)
    np.testing.assert_allclose(s_out.cpu().numpy(), s.cpu().numpy(), rtol=1e-5, atol=1e-12)
    assert rel(x, x_ref) < RTOL


def test_stream_matches_the_oracle(rlib, oracle, torch, case):
    ctx, lst, A, y, s, x_ref = case
    rp, col, val = A.to_numpy()
    yh = y.cpu().numpy()
    rows = np.nonzero(yh)[0]
    rp_m = np.concatenate([[0], np.cumsum(np.diff(rp)[rows])]).astype(np.int64)
    sel = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in rows])
    x0 = np.full(A.n, np.float32(1.0 / A.n), np.float32)
    want = oracle.mlem(rows.size, A.n, rp_m, col[sel], val[sel], yh[rows], s.cpu().numpy(), x0, NITER)
    x = torch.from_numpy(x0.copy()).cuda()
    ctx.mlem_stream(lst, 100, SEED, y, s, x, NITER, int(0.5 * (A.nnz * 8)))
    got = x.cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-4


def test_stream_rejects_bad_arguments(rlib, torch, case):
    ctx, lst, A, y, s, x_ref = case
    x = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    with pytest.raises(RuntimeError):
        ctx.mlem_stream(lst, 0, SEED, y, s, x, 2, 0)
    with pytest.raises(RuntimeError):
        ctx.mlem_stream(lst, 100, SEED, y, s, x, 2, -1)
    bad = lst.copy()
    bad[7] = ctx.n_channels  # out of range
    with pytest.raises(RuntimeError):
        ctx.mlem_stream(bad, 100, SEED, y, s, x, 2, 0)


def test_reco_host_falls_back_to_rebuilding_rows(rlib, torch, tmp_path):
    """raptr_reco_host in a process whose library memory is capped
    (RAPTR_DEVICE_MEMORY_LIMIT, 600 MB) below what the build, the matrix
    and its transpose need: the call keeps the rows that fit resident,
    rebuilds the others in every iteration, and returns the image of the
    uncapped call (1e-5; the back projections sum in another order)."""
    import os
    import subprocess
    import sys

    g = cfg.SMALL
    rng = np.random.default_rng(17)
    y = rng.poisson(3.0, g.n_channels).astype(np.float32)
    np.save(tmp_path / "y.npy", y)
    x_ref, st_ref = rlib.reco_host(g, y, 100, SEED, 6)
    assert st_ref["streamed_rows"] == 0
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "import raptr_b200 as R\n"
        "y = np.load(%r)\n"
        "x, st = R.reco_host(R.SMALL, y, 100, %d, 6)\n"
        "np.save(%r, x); print(st['streamed_rows'], st['nnz'])\n"
    ) % (root, str(tmp_path / "y.npy"), SEED, str(tmp_path / "x.npy"))
    env = dict(os.environ, RAPTR_DEVICE_MEMORY_LIMIT=str(600 << 20))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    streamed, resident_entries = (int(v) for v in r.stdout.split())
    assert 0 < streamed < g.n_channels and 0 < resident_entries < st_ref["nnz"]
    x = np.load(tmp_path / "x.npy")
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < RTOL
