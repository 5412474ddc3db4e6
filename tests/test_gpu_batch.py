"""Batched frames on the GPU: K reconstructions over one matrix in one
multi-right-hand-side pass must give, frame by frame, the single-frame
iteration's image (same matrix form), for every frame tile."""
import numpy as np
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu

SEED = 1251
K = 8
FRAME_RTOL = 1e-5  # batched vs single-frame image (relative L2); summation order differs


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


@pytest.fixture(scope="module")
def frames(rlib, torch):
    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    A = ctx.build(np.arange(g.n_channels, dtype=np.int32), 100, SEED)
    A.to_half()
    rp, col, val = A.to_numpy()
    from oracle import oracle as O

    rng = np.random.default_rng(3)
    xt = cfg.phantom(g, rods=False).astype(np.float64)
    Y = np.zeros((A.m, K), np.float32)
    for f in range(K):
        lam = O.spmv(0, A.m, A.n, rp, col, val, xt * np.exp(-0.05 * f), dtype=np.float64)
        Y[:, f] = cfg.poisson_measurement(lam, float(10 ** rng.uniform(5, 6.5)), seed=100 + f)
    return ctx, A, Y


@pytest.mark.parametrize("half", [False, True])
@pytest.mark.parametrize("tile", [4, 8])
def test_batch_equals_single_frames(rlib, torch, frames, half, tile):
    ctx, A, Y = frames
    n = A.n
    s = (rlib.sensitivity_half(A) if half else rlib.sensitivity(A))[1]
    Yd = torch.from_numpy(Y).cuda()
    X = torch.full((n, K), np.float32(1.0 / n), device="cuda")
    ctx.mlem_batch(A, Yd, s, X, 6, frame_tile=tile, half=half, use_graph=True)
    Xb = X.cpu().numpy()
    for f in (0, 3, K - 1):
        x = torch.full((n,), np.float32(1.0 / n), device="cuda")
        y = Yd[:, f].contiguous()
        if half:
            ctx.mlem_half(A, y, s, x, 6)
        else:
            ctx.mlem(A, y, s, x, 6)
        x = x.cpu().numpy()
        assert np.linalg.norm(Xb[:, f] - x) / np.linalg.norm(x) < FRAME_RTOL
        assert abs(float(Xb[:, f].sum()) - 1.0) < 1e-5


def test_batch_graph_timing_and_autotune(rlib, torch, frames):
    ctx, A, Y = frames
    n = A.n
    s = rlib.sensitivity_half(A)[1]
    Yd = torch.from_numpy(Y).cuda()
    X0 = torch.full((n, K), np.float32(1.0 / n), device="cuda")
    best, ms = ctx.batch_autotune(A, Yd, s, X0)
    assert best in ms and set(ms) == {4, 8}
    assert torch.all(X0 == np.float32(1.0 / n))  # the autotuner leaves the images alone
    Xg = X0.clone()
    ctx.mlem_batch(A, Yd, s, Xg, 3, frame_tile=best, use_graph=True)
    Xt = X0.clone()
    kt = ctx.mlem_batch(A, Yd, s, Xt, 3, frame_tile=best, use_graph=False, kernel_times=True)
    assert kt.shape == (3, 2) and np.all(kt > 0)
    assert torch.equal(Xg, Xt)


def test_batch_rejects_bad_tile(rlib, torch, frames):
    ctx, A, Y = frames
    n = A.n
    s = rlib.sensitivity(A)[1]
    X = torch.full((n, K), np.float32(1.0 / n), device="cuda")
    with pytest.raises(RuntimeError):
        ctx.mlem_batch(A, torch.from_numpy(Y).cuda(), s, X, 1, frame_tile=16)  # does not divide 8
    with pytest.raises(RuntimeError):
        ctx.mlem_batch(A, torch.from_numpy(Y).cuda(), s, X, 1, frame_tile=6)
