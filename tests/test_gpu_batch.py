"""Batched frames on the GPU: K reconstructions over one matrix in one
multi-right-hand-side pass must give, frame by frame, the single-frame
iteration's image (same matrix form), for every frame tile.  At 64 frames
of uneven counts (the dynamic-PET form: one geometry, counts log-uniform
in [1e5, 1e8]) every tile the autotuner can pick is checked, in FP32 and
FP16, against the single-frame iteration and against the CPU FP64 oracle
(src/tests/reco.cu:229-321 in FP64 over the measured rows)."""
import numpy as np
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu

SEED = 1251
K = 12
FRAME_RTOL = 1e-5  # batched vs single-frame image (relative L2); summation order differs
F64_RTOL = {False: 1e-4, True: 1e-3}  # vs the FP64 oracle: FP32 matrix, FP16 matrix
K64 = 64
NIT64 = 6


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
@pytest.mark.parametrize("tile", [4, 8, 64])
def test_batch_equals_single_frames(rlib, torch, frames, half, tile):
    """Each frame of the batch equals its own single-frame iteration; with
    tile 64 the 12 frames run as tiles of 8 and 4 narrower than the batch
    (their images gathered from a compact copy, as at tiles 4 and 8)."""
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
    assert best in ms and set(ms) == {4, 8, 16, 32, 64}
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
        ctx.mlem_batch(A, torch.from_numpy(Y).cuda(), s, X, 1, frame_tile=6)
    X6 = torch.full((n, 6), np.float32(1.0 / n), device="cuda")
    with pytest.raises(RuntimeError):  # not a multiple of 4 frames
        ctx.mlem_batch(A, torch.from_numpy(np.ascontiguousarray(Y[:, :6])).cuda(), s, X6, 1, frame_tile=4)


# ---------------------------------------------------------------- 64 frames


@pytest.fixture(scope="module")
def frames64(rlib, torch):
    """64 frames of the C1 geometry: x_true under a seeded exponential
    washout (rate uniform in [0.01, 0.1] per frame), counts log-uniform in
    [1e5, 1e8]."""
    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    A = ctx.build(np.arange(g.n_channels, dtype=np.int32), 100, SEED)
    A.to_half()
    rp, col, val = A.to_numpy()
    from oracle import oracle as O

    rng = np.random.default_rng(64)
    rate = rng.uniform(0.01, 0.1)
    xt = cfg.phantom(g, rods=False).astype(np.float64)
    lam = O.spmv(0, A.m, A.n, rp, col, val, xt, dtype=np.float64)
    Y = np.zeros((A.m, K64), np.float32)
    for f in range(K64):
        counts = 10 ** rng.uniform(5, 8)
        Y[:, f] = cfg.poisson_measurement(lam * np.exp(-rate * f), counts, seed=1000 + f)
    return ctx, A, Y, (rp, col, val)


@pytest.fixture(scope="module")
def single64(rlib, torch, frames64):
    """Single-frame images of all 64 frames, FP32 and FP16 matrix."""
    ctx, A, Y, _ = frames64
    n = A.n
    out = {}
    for half in (False, True):
        s = (rlib.sensitivity_half(A) if half else rlib.sensitivity(A))[1]
        imgs = np.zeros((n, K64), np.float32)
        for f in range(K64):
            x = torch.full((n,), np.float32(1.0 / n), device="cuda")
            y = torch.from_numpy(np.ascontiguousarray(Y[:, f])).cuda()
            (ctx.mlem_half if half else ctx.mlem)(A, y, s, x, NIT64)
            imgs[:, f] = x.cpu().numpy()
        out[half] = imgs
    return out


@pytest.fixture(scope="module")
def oracle64(frames64):
    """FP64 oracle images of frames 0, 31 and 63 over their measured rows,
    with the FP64 sensitivity of all rows."""
    from oracle import oracle as O

    ctx, A, Y, (rp, col, val) = frames64
    s = O.column_sums_f64(A.m, A.n, rp, col, val)
    s /= s.sum()
    out = {}
    for f in (0, 31, K64 - 1):
        rows = np.nonzero(Y[:, f])[0]
        rp_m = np.concatenate([[0], np.cumsum(np.diff(rp)[rows])]).astype(np.int64)
        sel = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in rows])
        x0 = np.full(A.n, 1.0 / A.n)
        out[f] = O.mlem(rows.size, A.n, rp_m, col[sel], val[sel], Y[rows, f].astype(np.float64), s, x0, NIT64,
                        dtype=np.float64)
    return out


@pytest.mark.parametrize("half", [False, True])
@pytest.mark.parametrize("tile", [4, 8, 16, 32, 64])
def test_batch64_every_tile(rlib, torch, frames64, single64, oracle64, half, tile):
    ctx, A, Y, _ = frames64
    n = A.n
    s = (rlib.sensitivity_half(A) if half else rlib.sensitivity(A))[1]
    X = torch.full((n, K64), np.float32(1.0 / n), device="cuda")
    ctx.mlem_batch(A, torch.from_numpy(Y).cuda(), s, X, NIT64, frame_tile=tile, half=half, use_graph=True)
    Xb = X.cpu().numpy()
    ref = single64[half]
    for f in range(K64):
        err = np.linalg.norm(Xb[:, f] - ref[:, f]) / np.linalg.norm(ref[:, f])
        assert err < FRAME_RTOL, f"frame {f}: rel L2 {err:.2e} against the single-frame iteration"
        assert abs(float(Xb[:, f].sum()) - 1.0) < 1e-5
    for f, want in oracle64.items():
        err = np.linalg.norm(Xb[:, f].astype(np.float64) - want) / np.linalg.norm(want)
        assert err < F64_RTOL[half], f"frame {f}: rel L2 {err:.2e} against the FP64 oracle"


def test_batch64_autotune_covers_every_tile(rlib, torch, frames64):
    ctx, A, Y, _ = frames64
    n = A.n
    s = rlib.sensitivity_half(A)[1]
    X0 = torch.full((n, K64), np.float32(1.0 / n), device="cuda")
    best, ms = ctx.batch_autotune(A, torch.from_numpy(Y).cuda(), s, X0)
    assert set(ms) == {4, 8, 16, 32, 64} and best in ms
    assert all(v > 0 for v in ms.values())
    assert torch.all(X0 == np.float32(1.0 / n))


def test_batch_back_pass_in_row_block_groups(rlib, torch):
    """Frames whose ratios of one tile exceed L2 (here 30 angles of the full
    geometry, 856,830 rows: 219 MB of ratios per 64-frame tile, 110 MB per
    32-frame tile) run the back pass in groups of row blocks with partial
    sums; every frame still equals the single-frame iteration."""
    g = cfg.FULL
    per = g.n0z * g.n0y * g.n1z * g.n1y
    lst = np.concatenate([np.arange(a * per, (a + 1) * per) for a in range(0, g.na, 6)]).astype(np.int32)
    ctx = rlib.Context(g, 0)
    A = ctx.build(lst, 200, SEED)
    A.to_half()
    xt = torch.from_numpy(cfg.phantom(g, rods=True)).cuda()
    lam = rlib.spmv(rlib.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, xt).cpu().numpy()
    rng = np.random.default_rng(9)
    Y = np.stack([cfg.poisson_measurement(lam, 10 ** rng.uniform(5, 7), seed=700 + f) for f in range(K64)], 1)
    Y = np.ascontiguousarray(Y, np.float32)
    s = rlib.sensitivity_half(A)[1]
    Yd = torch.from_numpy(Y).cuda()
    n = A.n
    ref = np.zeros((n, K64), np.float32)
    for f in range(K64):
        x = torch.full((n,), np.float32(1.0 / n), device="cuda")
        ctx.mlem_half(A, Yd[:, f].contiguous(), s, x, 3)
        ref[:, f] = x.cpu().numpy()
    for tile in (32, 64):
        X = torch.full((n, K64), np.float32(1.0 / n), device="cuda")
        ctx.mlem_batch(A, Yd, s, X, 3, frame_tile=tile, half=True, use_graph=True)
        Xb = X.cpu().numpy()
        for f in range(K64):
            err = np.linalg.norm(Xb[:, f] - ref[:, f]) / np.linalg.norm(ref[:, f])
            assert err < FRAME_RTOL, f"tile {tile}, frame {f}: rel L2 {err:.2e}"
