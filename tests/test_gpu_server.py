"""The serving loop on the GPU: every result is the same whether the
request ran alone or among others of mixed geometry (continuous batching),
matches the FP16 single-frame iteration and the FP64 oracle iteration,
and the matrix cache evicts within its byte budget."""
import numpy as np
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu

NRAYS, SEED = 50, 1251
MIX_RTOL = 1e-5    # alone vs in the mix, and vs the single-frame FP16 iteration
F64_RTOL = 1e-3    # vs the FP64 iteration on the FP32 matrix
MINI = cfg.epet_geometry(30, 0.002, 4, 45.0)


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def measurement(rlib, torch, g, counts, seed):
    ctx = rlib.Context(g, 0)
    A = ctx.build(np.arange(g.n_channels, dtype=np.int32), NRAYS, SEED)
    xt = torch.from_numpy(cfg.phantom(g, rods=False)).cuda()
    lam = rlib.spmv(rlib.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, xt).cpu().numpy()
    return cfg.poisson_measurement(lam, counts, seed)


@pytest.fixture(scope="module")
def jobs(rlib, torch):
    out = []
    for i, (g, it) in enumerate([(cfg.SMALL, 5), (MINI, 7), (cfg.SMALL, 9), (MINI, 4), (cfg.SMALL, 6), (MINI, 8)]):
        out.append((g, it, measurement(rlib, torch, g, 10 ** (5 + 0.4 * i), 40 + i)))
    return out


def rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))


def test_alone_and_in_the_mix(rlib, torch, jobs):
    srv = rlib.Server(0, hbm_budget_bytes=20 << 30)
    alone = []
    for g, it, y in jobs:
        rid = srv.submit(g, y, it, NRAYS, SEED)
        x, st = srv.wait(rid, g.n_voxels)
        assert st["iterations"] == it
        alone.append(x)
    ids = [srv.submit(g, y, it, NRAYS, SEED) for g, it, y in jobs]
    frames = []
    for (g, it, y), rid, xa in zip(jobs, ids, alone):
        x, st = srv.wait(rid, g.n_voxels)
        assert rel(x, xa) < MIX_RTOL
        assert abs(float(x.sum()) - 1.0) < 1e-5
        frames.append(st["frames_max"])
    assert max(frames) >= 2  # requests of one geometry did share a batch
    s = srv.stats()
    assert s["builds"] == 2 and s["completed"] == 2 * len(jobs) and s["queued"] == 0 and s["running"] == 0
    srv.close()


def test_matches_single_frame_and_fp64(rlib, torch, jobs):
    g, it, y = jobs[0]
    srv = rlib.Server(0, hbm_budget_bytes=20 << 30)
    x, _ = srv.wait(srv.submit(g, y, it, NRAYS, SEED), g.n_voxels)
    srv.close()
    ctx = rlib.Context(g, 0)
    A = ctx.build(np.arange(g.n_channels, dtype=np.int32), NRAYS, SEED)
    A.to_half()
    yd = torch.from_numpy(y).cuda()
    h64, h32 = rlib.sensitivity_half(A)
    xh = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    ctx.mlem_half(A, yd, h32, xh, it)
    assert rel(x, xh.double().cpu().numpy()) < MIX_RTOL
    s64, _ = rlib.sensitivity(A)
    x64 = torch.full((A.n,), 1.0 / A.n, dtype=torch.float64, device="cuda")
    ctx.mlem_f64(A, yd, s64 / s64.sum(), x64, it)
    assert rel(x, x64.cpu().numpy()) < F64_RTOL


def test_cache_evicts_within_budget(rlib, torch, jobs):
    # room for one of the two matrices (by the pre-build estimate) at a time
    srv = rlib.Server(0, hbm_budget_bytes=int(1.45e9))
    ref = {}
    for g, it, y in jobs[:4]:
        x, st = srv.wait(srv.submit(g, y, it, NRAYS, SEED), g.n_voxels)
        key = (g.n_voxels, it)
        ref[key] = x
    s = srv.stats()
    assert s["evictions"] >= 1 and s["builds"] >= 3
    assert s["resident_bytes"] <= int(1.45e9)
    # results do not depend on rebuilds
    srv2 = rlib.Server(0, hbm_budget_bytes=20 << 30)
    for g, it, y in jobs[:4]:
        x, _ = srv2.wait(srv2.submit(g, y, it, NRAYS, SEED), g.n_voxels)
        assert rel(x, ref[(g.n_voxels, it)]) < MIX_RTOL
    srv.close()
    srv2.close()


def test_budget_too_small_and_timeout(rlib, torch, jobs):
    g, it, y = jobs[0]
    srv = rlib.Server(0, hbm_budget_bytes=1 << 20)
    rid = srv.submit(g, y, it, NRAYS, SEED)
    with pytest.raises(RuntimeError):
        srv.wait(rid, g.n_voxels)
    srv.close()
    srv = rlib.Server(0, hbm_budget_bytes=20 << 30)
    rid = srv.submit(g, y, 40, NRAYS, SEED)
    with pytest.raises(RuntimeError):
        srv.wait(rid, g.n_voxels, timeout_ms=0)  # still queued or running
    x, st = srv.wait(rid, g.n_voxels)
    assert st["iterations"] == 40
    with pytest.raises(RuntimeError):
        srv.wait(rid, g.n_voxels)  # already collected
    with pytest.raises(ValueError):
        srv.submit(g, y[:-1], 3, NRAYS, SEED)
    srv.close()


def test_many_requests_join_and_leave(rlib, torch):
    """50 requests of one geometry: 40 submitted at once (batches above 32
    frames), 10 more while those run (they join the running batch).  Every
    result equals the same request run alone on the same server (same cached
    matrix) to 1e-5, and the single-frame FP16 iteration on a matrix built
    apart to 1e-4 (the two builds' values differ in their last bits, which
    60-120 iterations carry further than the 1e-5 of a few iterations)."""
    g = MINI
    ctx = rlib.Context(g, 0)
    A = ctx.build(np.arange(g.n_channels, dtype=np.int32), NRAYS, SEED)
    xt = torch.from_numpy(cfg.phantom(g, rods=False)).cuda()
    lam = rlib.spmv(rlib.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, xt).cpu().numpy()
    rng = np.random.default_rng(50)
    reqs = []
    for i in range(50):
        it = int(rng.integers(60, 120)) if i < 40 else int(rng.integers(3, 12))
        if i == 0:
            it = 2  # finishes first: the cue for the second wave
        reqs.append((it, cfg.poisson_measurement(lam, 10 ** rng.uniform(5, 7), 500 + i)))
    A.to_half()
    h32 = rlib.sensitivity_half(A)[1]
    want = []
    for it, y in reqs:
        x = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
        ctx.mlem_half(A, torch.from_numpy(y).cuda(), h32, x, it)
        want.append(x.double().cpu().numpy())
    srv = rlib.Server(0, hbm_budget_bytes=20 << 30)
    ids = [srv.submit(g, y, it, NRAYS, SEED) for it, y in reqs[:40]]
    x0, st0 = srv.wait(ids[0], g.n_voxels)
    running_before = srv.stats()["running"]
    ids += [srv.submit(g, y, it, NRAYS, SEED) for it, y in reqs[40:]]
    out = [(x0, st0)] + [srv.wait(rid, g.n_voxels) for rid in ids[1:]]
    assert running_before > 0  # the second wave arrived while the first ran
    alone = [srv.wait(srv.submit(g, y, it, NRAYS, SEED), g.n_voxels) for it, y in reqs]
    srv.close()
    frames = []
    for (it, _), w, (x, st), (xa, sta) in zip(reqs, want, out, alone):
        assert st["iterations"] == it and sta["iterations"] == it and sta["frames_max"] == 1
        assert rel(x, xa.astype(np.float64)) < MIX_RTOL
        assert rel(x, w) < 1e-4
        assert abs(float(x.sum()) - 1.0) < 1e-5
        frames.append(st["frames_max"])
    assert max(frames[:40]) > 32  # batches above 32 frames ran
    assert min(frames[40:]) > 1   # the late requests ran beside others
