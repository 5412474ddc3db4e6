"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bars: bit-exact for integer/index work (candidates, CSR structure, ray
endpoints); matrix values within 1e-5 relative of the oracle given identical
rays (the GPU sums rays in a different order); MLEM images within 1e-4
relative L2 of the FP32 oracle.
"""
import numpy as np
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu

SEED = 1251
VAL_RTOL = 1e-5
IMG_RTOL = 1e-4


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


@pytest.fixture(scope="module")
def ctx_small(rlib, torch):
    return rlib.Context(cfg.SMALL, 0)


@pytest.fixture(scope="module")
def ctx_full(rlib, torch):
    return rlib.Context(cfg.FULL, 0)


def assert_rows_equal(rp_g, col_g, val_g, rp_o, col_o, val_o, rtol=VAL_RTOL):
    assert np.array_equal(rp_g, rp_o), "row pointers differ"
    assert np.array_equal(col_g, col_o), "columns differ"
    if val_o.size:
        err = np.abs(val_g.astype(np.float64) - val_o) / np.maximum(np.abs(val_o.astype(np.float64)), 1e-30)
        assert err.max() <= rtol, f"max rel err {err.max()}"


# ---------------------------------------------------------------- rays

@pytest.mark.parametrize("which", ["small", "full", "fine"])
def test_rays_bit_exact(rlib, oracle, torch, which):
    g = {"small": cfg.SMALL, "full": cfg.FULL, "fine": cfg.FINE}[which]
    ctx = rlib.Context(g, 0)
    rng = np.random.Generator(np.random.PCG64(11))
    lst = np.unique(np.concatenate([rng.integers(0, g.n_channels, 200), [0, g.n_channels - 1]])).astype(np.int32)
    got = ctx.rays(lst, 64, SEED).cpu().numpy()
    want = oracle.rays(g, lst, 64, SEED)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


# ---------------------------------------------------------------- candidates

def test_workqueue_matches_reference_golden(rlib, golden, ctx_small):
    c, v, cur = ctx_small.workqueue(golden["small_list"], max_out=1 << 20)
    assert np.array_equal(c.cpu().numpy(), golden["small_cnl"])
    assert np.array_equal(v.cpu().numpy(), golden["small_vxl"])
    assert cur == (golden["small_list"].size, 0)


def test_workqueue_cursor_chunks_match_reference(rlib, golden, ctx_small):
    cur = (0, 0)
    k = 0
    for n, cnt, want_cur in zip(golden["wq_sizes"], golden["wq_counts"], golden["wq_cursors"]):
        c, v, cur = ctx_small.workqueue(golden["wq_list"], cursor=cur, max_out=int(n))
        assert c.numel() == cnt
        assert np.array_equal(c.cpu().numpy(), golden["wq_cnl"][k:k + cnt])
        assert np.array_equal(v.cpu().numpy(), golden["wq_vxl"][k:k + cnt])
        assert tuple(cur) == tuple(want_cur)
        k += cnt


def test_workqueue_many_channels_bit_exact(rlib, oracle, ctx_small):
    g = cfg.SMALL
    lst = np.arange(0, g.n_channels, 41, dtype=np.int32)
    c, v, cur = ctx_small.workqueue(lst, max_out=lst.size * 6000)
    co, vo, curo = oracle.workqueue(g, lst)
    assert np.array_equal(c.cpu().numpy(), co) and np.array_equal(v.cpu().numpy(), vo)
    assert cur == curo


def test_workqueue_full_geometry_bit_exact(rlib, oracle, ctx_full):
    g = cfg.FULL
    rng = np.random.Generator(np.random.PCG64(5))
    lst = rng.integers(0, g.n_channels, 120).astype(np.int32)
    c, v, cur = ctx_full.workqueue(lst, max_out=lst.size * 20000)
    co, vo, curo = oracle.workqueue(g, lst)
    assert np.array_equal(c.cpu().numpy(), co) and np.array_equal(v.cpu().numpy(), vo)
    counts = ctx_full.candidate_counts(lst).cpu().numpy()
    assert np.array_equal(counts, oracle.candidate_counts(g, lst))


def test_workqueue_edge_cases(rlib, oracle, ctx_small):
    g = cfg.SMALL
    lst = np.array([7, 8], np.int32)
    # max_out = 0 leaves the cursor untouched
    c, v, cur = ctx_small.workqueue(lst, cursor=(1, 5), max_out=0)
    assert c.numel() == 0 and cur == (1, 5)
    # empty list
    c, v, cur = ctx_small.workqueue(np.zeros(0, np.int32), max_out=10)
    assert c.numel() == 0 and cur == (0, 0)
    # cursor in the middle of a row, and at the last voxel
    for start in [(0, 31000), (1, g.n_voxels - 1), (2, 0)]:
        c, v, cur = ctx_small.workqueue(lst, cursor=start, max_out=100000)
        co, vo, curo = oracle.workqueue(g, lst, cursor=start)
        assert np.array_equal(c.cpu().numpy(), co) and np.array_equal(v.cpu().numpy(), vo) and cur == curo
    # a limit that ends exactly at the last candidate of the first channel
    co, vo, _ = oracle.workqueue(g, lst[:1])
    c, v, cur = ctx_small.workqueue(lst, max_out=co.size)
    _, _, curo = oracle.workqueue(g, lst, max_out=co.size)
    assert cur == curo


# ---------------------------------------------------------------- system matrix

@pytest.fixture(scope="module")
def small_full_matrix(rlib, oracle, ctx_small):
    g = cfg.SMALL
    lst = np.arange(g.n_channels, dtype=np.int32)
    A = ctx_small.build(lst, 100, SEED)
    rp, col, val = oracle.sysmat(g, lst, 100, SEED, method=1)
    return A, (rp, col, val), lst


def test_sysmat_small_all_channels(small_full_matrix):
    A, (rp, col, val), lst = small_full_matrix
    assert A.m == lst.size and A.nnz == col.size
    assert_rows_equal(*A.to_numpy(), rp, col, val)


def test_sysmat_keep_zeros_matches_reference_golden(rlib, golden, ctx_small):
    A = ctx_small.build(golden["small_list"], 100, SEED, keep_zeros=True)
    rp, col, val = A.to_numpy()
    assert np.array_equal(np.repeat(golden["small_list"], np.diff(rp)), golden["small_cnl"])
    assert np.array_equal(col, golden["small_vxl"])
    want = golden["small_val"].astype(np.float64)
    assert np.all((val == 0) == (want == 0))
    nz = want != 0
    assert np.max(np.abs(val[nz] - want[nz]) / want[nz]) <= VAL_RTOL


def test_sysmat_full_geometry_golden_rows(rlib, golden, ctx_full):
    A = ctx_full.build(golden["full_list"], 64, SEED, keep_zeros=True)
    rp, col, val = A.to_numpy()
    assert np.array_equal(col, golden["full_vxl"])
    want = golden["full_val"].astype(np.float64)
    assert np.all((val == 0) == (want == 0))
    nz = want != 0
    assert np.max(np.abs(val[nz] - want[nz]) / want[nz]) <= VAL_RTOL


def test_sysmat_full_geometry_1000_rays(rlib, oracle, ctx_full):
    g = cfg.FULL
    rng = np.random.Generator(np.random.PCG64(8))
    lst = rng.integers(0, g.n_channels, 300).astype(np.int32)
    A = ctx_full.build(lst, 1000, SEED)
    assert_rows_equal(*A.to_numpy(), *oracle.sysmat(g, lst, 1000, SEED, method=1))


def test_sysmat_fine_geometry(rlib, oracle):
    g = cfg.FINE
    ctx = rlib.Context(g, 0)
    rng = np.random.Generator(np.random.PCG64(9))
    lst = rng.integers(0, g.n_channels, 60).astype(np.int32)
    A = ctx.build(lst, 1000, SEED)
    assert_rows_equal(*A.to_numpy(), *oracle.sysmat(g, lst, 1000, SEED, method=1))


def test_sysmat_anisotropic_offset_grid(rlib, oracle):
    # Origin, pitch and size differ per axis and the grid is off centre: the
    # walk's general step (origin selected per axis) against the oracle.
    g = cfg.Geometry(grid_o=(-0.061, -0.047, -0.039), grid_d=(0.002, 0.0025, 0.0018), grid_n=(60, 40, 48),
                     pos0x=-0.240, pos1x=0.240, na=12, n0z=13, n0y=13, n1z=13, n1y=13, da=15.0, segx=0.020,
                     segy=0.004, segz=0.004)
    ctx = rlib.Context(g, 0)
    rng = np.random.Generator(np.random.PCG64(10))
    lst = rng.integers(0, g.n_channels, 80).astype(np.int32)
    A = ctx.build(lst, 300, SEED)
    assert A.nnz > 0
    assert_rows_equal(*A.to_numpy(), *oracle.sysmat(g, lst, 300, SEED, method=1))


def test_sysmat_given_rays_with_axis_parallel_rays(rlib, oracle, torch, ctx_small):
    # Identical caller-supplied endpoints, including rays parallel to a plane
    # family, against the reference algorithm (method 0).
    g = cfg.SMALL
    lst = np.array([40000, 40001, 71234], np.int32)
    rays = oracle.rays(g, lst, 32, 5)
    rays[0, :, 4] = rays[0, :, 1]
    rays[1, :10, 5] = rays[1, :10, 2]
    A = ctx_small.build(lst, 32, 0, rays=torch.from_numpy(rays))
    assert_rows_equal(*A.to_numpy(), *oracle.sysmat(g, lst, 32, 0, rays_in=rays, method=0))


def test_sysmat_duplicate_and_unordered_list(rlib, oracle, ctx_small):
    g = cfg.SMALL
    lst = np.array([99, 5, 99, 142804, 0], np.int32)
    A = ctx_small.build(lst, 100, SEED)
    assert_rows_equal(*A.to_numpy(), *oracle.sysmat(g, lst, 100, SEED, method=1))


def test_sysmat_caller_buffers_two_phase(rlib, oracle, torch, ctx_small):
    g = cfg.SMALL
    lst = np.arange(1000, 1400, dtype=np.int32)
    rp_o, col_o, val_o = oracle.sysmat(g, lst, 100, SEED, method=1)
    rp = torch.empty(lst.size + 1, dtype=torch.int64, device="cuda")
    col = torch.empty(10, dtype=torch.int32, device="cuda")
    val = torch.empty(10, dtype=torch.float32, device="cuda")
    st, nnz = ctx_small.build_into(lst, 100, SEED, rp, col, val)
    assert st == rlib.RAPTR_ERR_CAPACITY and nnz == col_o.size
    assert np.array_equal(rp.cpu().numpy(), rp_o)
    col = torch.empty(nnz, dtype=torch.int32, device="cuda")
    val = torch.empty(nnz, dtype=torch.float32, device="cuda")
    st, nnz2 = ctx_small.build_into(lst, 100, SEED, rp, col, val)
    assert st == 0 and nnz2 == nnz
    assert_rows_equal(rp.cpu().numpy(), col.cpu().numpy(), val.cpu().numpy(), rp_o, col_o, val_o)


def test_sysmat_empty_list(rlib, ctx_small):
    A = ctx_small.build(np.zeros(0, np.int32), 100, SEED)
    assert A.m == 0 and A.nnz == 0 and A.row_ptr.cpu().tolist() == [0]


def test_invalid_arguments_raise(rlib, ctx_small):
    with pytest.raises(rlib.RaptrError):
        ctx_small.build(np.array([1], np.int32), 0, SEED)


# ---------------------------------------------------------------- SpMV / ops

def test_spmv_forward_and_back(rlib, oracle, torch, small_full_matrix):
    A, (rp, col, val), lst = small_full_matrix
    g = cfg.SMALL
    rng = np.random.Generator(np.random.PCG64(2))
    x = rng.random(g.n_voxels).astype(np.float32)
    e = rng.random(A.m).astype(np.float32)
    yt = rlib.spmv(rlib.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, torch.from_numpy(x).cuda()).cpu().numpy()
    want = oracle.spmv(0, A.m, A.n, rp, col, val, x.astype(np.float64), dtype=np.float64)
    assert np.max(np.abs(yt - want) / np.maximum(np.abs(want), 1e-30)) < 1e-5
    c0 = rng.random(g.n_voxels).astype(np.float32)
    c = rlib.spmv(rlib.OP_T, A.m, A.n, A.row_ptr, A.col, A.val, torch.from_numpy(e).cuda(), alpha=2.0, beta=0.5,
                  y=torch.from_numpy(c0.copy()).cuda()).cpu().numpy()
    want = oracle.spmv(1, A.m, A.n, rp, col, val, e.astype(np.float64), alpha=2.0, beta=0.5,
                       y=c0.astype(np.float64), dtype=np.float64)
    assert np.max(np.abs(c - want) / np.maximum(np.abs(want), 1e-30)) < 1e-5


def test_mlem_operations_known_answers(rlib, golden, torch):
    n = 10
    A = torch.tensor(((np.arange(n) + 1) ** 2).astype(np.float32)).cuda()
    B = torch.full((n,), 10.0, device="cuda")
    Cc = torch.arange(1, n + 1, dtype=torch.float32, device="cuda")
    D = torch.zeros(n, device="cuda")
    rlib.divides(D, A, Cc)
    assert np.array_equal(D.cpu().numpy(), golden["mlem_divides"])
    rlib.divides_multiplies(D, A, B, Cc)
    assert np.array_equal(D.cpu().numpy(), golden["mlem_divmul"])
    assert rlib.vsum(D) == 550.0
    rlib.scales(D, float(np.float32(1.0 / 550.0)))
    assert np.array_equal(D.cpu().numpy(), golden["mlem_scaled"])
    z = torch.tensor([0.0, 2.0], device="cuda")
    rlib.divides_multiplies(D[:2], torch.tensor([2.0, 3.0], device="cuda"), torch.tensor([5.0, 7.0], device="cuda"), z)
    assert D[:2].cpu().tolist() == [10.0, 10.5]


def test_coo2csr_and_ecsr_known_answers(rlib, torch):
    rows = torch.tensor([0, 1, 1, 1, 2, 2, 3, 3, 3], dtype=torch.int32, device="cuda")
    assert rlib.coo2csr(rows, 4).cpu().tolist() == [0, 1, 4, 6, 9]
    e = rlib.csr2ecsr(torch.tensor([2, 4, 6], dtype=torch.int32, device="cuda"),
                      torch.tensor([0, 0, 0, 3, 3, 3, 3, 5], dtype=torch.int64, device="cuda"))
    assert e.cpu().tolist() == [0, 3, 3, 5]


def sensitivity_csc(rlib, torch, A):
    """raptr_sensitivity_csc over a transpose of A's arrays (caller buffers,
    so that the shared matrix keeps no transpose)."""
    cp, _, tv = rlib.csr_transpose(A.m, A.n, A.row_ptr, A.col, A.val)
    s64 = torch.empty(A.n, dtype=torch.float64, device="cuda")
    s32 = torch.empty(A.n, dtype=torch.float32, device="cuda")
    rlib._check(rlib.lib().raptr_sensitivity_csc(A.n, cp.data_ptr(), tv.data_ptr(), s64.data_ptr(), s32.data_ptr(),
                                                 None))
    return s64, s32


@pytest.mark.parametrize("through", ["rows", "transpose"])
def test_sensitivity_fp64(rlib, oracle, torch, small_full_matrix, through):
    A, (rp, col, val), lst = small_full_matrix
    assert not A.has_transpose
    if through == "transpose":
        s64, s32 = sensitivity_csc(rlib, torch, A)
    else:
        s64, s32 = rlib.sensitivity(A)
    s64 = s64.cpu().numpy()
    # against the column sums of the same (GPU) values: FP64 sums in another order
    rp_g, col_g, val_g = A.to_numpy()
    want = oracle.column_sums_f64(A.m, A.n, rp_g, col_g, val_g)
    assert np.max(np.abs(s64 - want)) <= 1e-12 * want.max()
    np.testing.assert_allclose(s32.cpu().numpy(), (want / want.sum()).astype(np.float32), rtol=1e-6, atol=1e-12)
    # against the oracle's matrix: values agree to 1e-5, so do the sums
    want_o = oracle.column_sums_f64(A.m, A.n, rp, col, val)
    assert np.max(np.abs(s64 - want_o)) <= 1e-5 * want_o.max()
    if through == "transpose":
        # no atomics: the same bits on every run
        again, _ = sensitivity_csc(rlib, torch, A)
        assert np.array_equal(again.cpu().numpy(), s64)


# ---------------------------------------------------------------- MLEM

@pytest.fixture(scope="module")
def small_measurement(small_full_matrix):
    A, (rp, col, val), lst = small_full_matrix
    g = cfg.SMALL
    xt = cfg.phantom(g, rods=False)
    from oracle import oracle as O

    lam = O.spmv(0, A.m, A.n, rp, col, val, xt.astype(np.float64), dtype=np.float64)
    y = cfg.poisson_measurement(lam, 2e6, seed=7)
    return y


def test_mlem_matches_oracle(rlib, oracle, torch, ctx_small, small_full_matrix, small_measurement):
    A, (rp, col, val), lst = small_full_matrix
    y = small_measurement
    meas = y != 0
    # the oracle uses only measured rows (the reference's matrix has no others)
    rows = np.nonzero(meas)[0]
    rp_m = np.concatenate([[0], np.cumsum(np.diff(rp)[rows])]).astype(np.int64)
    col_m = np.concatenate([col[rp[r]:rp[r + 1]] for r in rows]).astype(np.int32)
    val_m = np.concatenate([val[rp[r]:rp[r + 1]] for r in rows]).astype(np.float32)
    s_all = oracle.column_sums_f64(A.m, A.n, rp, col, val)
    s = (s_all / s_all.sum()).astype(np.float32)
    n = A.n
    x0 = np.full(n, np.float32(1.0 / n), np.float32)
    want32 = oracle.mlem(rows.size, n, rp_m, col_m, val_m, y[rows], s, x0, 20)
    want64 = oracle.mlem(rows.size, n, rp_m, col_m, val_m, y[rows].astype(np.float64), s.astype(np.float64),
                         x0.astype(np.float64), 20, dtype=np.float64)
    for use_graph, transposed in ((False, False), (True, False), (False, True), (True, True)):
        if transposed and not A.has_transpose:
            A.transpose()
        assert A.has_transpose == transposed
        x = torch.from_numpy(x0.copy()).cuda()
        ll = ctx_small.mlem(A, torch.from_numpy(y).cuda(), torch.from_numpy(s).cuda(), x, 20, use_graph=use_graph,
                            loglik=True)
        x = x.cpu().numpy()
        assert np.linalg.norm(x - want32) / np.linalg.norm(want32) < IMG_RTOL
        assert np.linalg.norm(x - want64) / np.linalg.norm(want64) < IMG_RTOL
        assert abs(float(x.sum()) - 1.0) < 1e-5
        assert np.all(np.diff(ll) >= -1e-6 * abs(ll[-1]))  # MLEM never decreases the likelihood


def test_mlem_full_geometry_four_angles_50_iterations(rlib, oracle, torch, ctx_full):
    """The full workload's iteration on a row subset of its geometry: all
    channels of four angles (0, 46, 90 and 134 degrees: x-slab, diagonal and
    z-slab rows) of the 70^3 grid, 1000 rays, rod phantom, 50 iterations
    through the transpose in back-projection order (the benchmarked path),
    against the FP32 and FP64 oracles (src/tests/reco.cu:229-321) at 1e-4
    relative L2.  A row sample is first checked against the oracle's own
    rows."""
    g = cfg.FULL
    per = g.n0z * g.n0y * g.n1z * g.n1y
    lst = np.concatenate([np.arange(a * per, (a + 1) * per) for a in (0, 23, 45, 67)]).astype(np.int32)
    A = ctx_full.build(lst, 1000, SEED)
    rp, col, val = A.to_numpy()
    sample = np.arange(0, lst.size, lst.size // 16)
    rp_o, col_o, val_o = oracle.sysmat(g, lst[sample], 1000, SEED, method=1)
    rp_s = np.concatenate([[0], np.cumsum(np.diff(rp)[sample])]).astype(np.int64)
    sel = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in sample])
    assert_rows_equal(rp_s, col[sel], val[sel], rp_o, col_o, val_o)
    xt = cfg.phantom(g, rods=True).astype(np.float64)
    lam = oracle.spmv(0, A.m, A.n, rp, col, val, xt, dtype=np.float64)
    y = cfg.poisson_measurement(lam, 1e8 * lst.size / g.n_channels, seed=70)
    rows = np.nonzero(y)[0]
    rp_m = np.concatenate([[0], np.cumsum(np.diff(rp)[rows])]).astype(np.int64)
    sel = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in rows])
    col_m, val_m = col[sel], val[sel]
    s_all = oracle.column_sums_f64(A.m, A.n, rp, col, val)
    s = (s_all / s_all.sum()).astype(np.float32)
    x0 = np.full(A.n, np.float32(1.0 / A.n), np.float32)
    want32 = oracle.mlem(rows.size, A.n, rp_m, col_m, val_m, y[rows], s, x0, 50)
    want64 = oracle.mlem(rows.size, A.n, rp_m, col_m, val_m, y[rows].astype(np.float64), s.astype(np.float64),
                         x0.astype(np.float64), 50, dtype=np.float64)
    A.transpose()
    x = torch.from_numpy(x0.copy()).cuda()
    ctx_full.mlem(A, torch.from_numpy(y).cuda(), torch.from_numpy(s).cuda(), x, 50, use_graph=True)
    x = x.cpu().numpy()
    assert np.linalg.norm(x - want32) / np.linalg.norm(want32) < IMG_RTOL
    assert np.linalg.norm(x - want64) / np.linalg.norm(want64) < IMG_RTOL
    assert abs(float(x.sum()) - 1.0) < 1e-5


def channel_order_keys(g, cnl):
    """Back-projection order key of channels: (angle, z0+z1, y0+y1, z0-z1,
    y0-y1), y1 fastest in the channel id."""
    c = np.asarray(cnl, np.int64)
    y1 = c % g.n1y
    z1 = (c // g.n1y) % g.n1z
    y0 = (c // (g.n1y * g.n1z)) % g.n0y
    z0 = (c // (g.n1y * g.n1z * g.n0y)) % g.n0z
    a = c // (g.n1y * g.n1z * g.n0y * g.n0z)
    sz, sy = g.n0z + g.n1z - 1, g.n0y + g.n1y - 1
    return (((a * sz + z0 + z1) * sy + y0 + y1) * sz + z0 - z1 + g.n1z - 1) * sy + y0 - y1 + g.n1y - 1


def csc_reference(m, n, rp, col, val):
    """CSC with rows ascending within each column (numpy stable sort)."""
    rows = np.repeat(np.arange(m), np.diff(rp))
    o = np.argsort(col, kind="stable")
    cp = np.zeros(n + 1, np.int64)
    cp[1:] = np.cumsum(np.bincount(col, minlength=n))
    return cp, rows[o].astype(np.int32), val[o]


def test_transpose_is_csc_of_the_matrix(rlib, torch, small_full_matrix):
    A, _, lst = small_full_matrix
    A.transpose()
    rp, col, val = A.to_numpy()
    cp = A.col_ptr.cpu().numpy()
    ri = A.row_idx.cpu().numpy()
    tv = A.tval.cpu().numpy()
    # the rows come in the back-projection order of their channels
    order = A.row_order.cpu().numpy()
    rank = A.row_rank.cpu().numpy()
    assert np.array_equal(order, np.argsort(channel_order_keys(cfg.SMALL, lst), kind="stable"))
    assert np.array_equal(rank[order], np.arange(A.m))
    # positions ascend within each column, and mapped back to rows the
    # transpose is exactly the CSC of the matrix in that order
    pos_rows = rank[np.repeat(np.arange(A.m), np.diff(rp))]
    o = np.lexsort((pos_rows, col))
    assert np.array_equal(cp, np.concatenate([[0], np.cumsum(np.bincount(col, minlength=A.n))]))
    assert np.array_equal(ri, pos_rows[o])
    assert np.array_equal(tv.view(np.uint32), val[o].view(np.uint32))
    assert np.array_equal(order[ri], np.repeat(np.arange(A.m), np.diff(rp))[o])


def test_csr_transpose_is_deterministic_and_sorted(rlib, torch, small_full_matrix):
    A, _, _ = small_full_matrix
    rp, col, val = A.to_numpy()
    cp_ref, ri_ref, tv_ref = csc_reference(A.m, A.n, rp, col, val)
    for _ in range(2):
        cp, ri, tv = rlib.csr_transpose(A.m, A.n, A.row_ptr, A.col, A.val)
        assert np.array_equal(cp.cpu().numpy(), cp_ref)
        assert np.array_equal(ri.cpu().numpy(), ri_ref)
        assert np.array_equal(tv.cpu().numpy().view(np.uint32), tv_ref.view(np.uint32))


def test_csr_transpose_in_a_given_order(rlib, torch, small_full_matrix):
    A, _, _ = small_full_matrix
    rp, col, val = A.to_numpy()
    order = np.random.default_rng(5).permutation(A.m).astype(np.int32)
    rank = np.empty(A.m, np.int64)
    rank[order] = np.arange(A.m)
    cp, pos, tv = rlib.csr_transpose_ordered(A.m, A.n, A.row_ptr, A.col, A.val, torch.from_numpy(order).cuda())
    pos_rows = rank[np.repeat(np.arange(A.m), np.diff(rp))]
    o = np.lexsort((pos_rows, col))
    assert np.array_equal(pos.cpu().numpy(), pos_rows[o])
    assert np.array_equal(tv.cpu().numpy().view(np.uint32), val[o].view(np.uint32))
    # back projection through it reads e in that order
    e = torch.rand(A.m, device="cuda")
    c_nat = rlib.spmv(rlib.OP_T, A.m, A.n, A.row_ptr, A.col, A.val, e)
    c = torch.zeros(A.n, device="cuda")
    rlib.lib().raptr_mlem_back(A.n, cp.data_ptr(), pos.data_ptr(), tv.data_ptr(),
                               e[torch.from_numpy(order).long().cuda()].contiguous().data_ptr(), c.data_ptr(), None)
    assert torch.allclose(c, c_nat, rtol=1e-5, atol=1e-6 * float(c_nat.abs().max()))
    # a bad order entry is an error, not a fault
    bad = order.copy()
    bad[3] = A.m + 7
    with pytest.raises(RuntimeError):
        rlib.csr_transpose_ordered(A.m, A.n, A.row_ptr, A.col, A.val, torch.from_numpy(bad).cuda())


def test_mlem_half_steps_equal_full_iteration(rlib, torch, ctx_small, small_full_matrix, small_measurement):
    A, _, _ = small_full_matrix
    A.transpose()
    y = torch.from_numpy(small_measurement).cuda()
    s64, s = rlib.sensitivity(A)
    n = A.n
    x1 = torch.full((n,), 1.0 / n, device="cuda")
    x2 = x1.clone()
    x3 = x1.clone()
    ctx_small.mlem(A, y, s, x1, 3, use_graph=False)
    c = torch.zeros(n, device="cuda")
    e = torch.zeros(A.m, device="cuda")
    acc = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(3):
        rlib.mlem_project(A, y, x2, c)
        rlib.mlem_update(x2, c, s, acc)
        rlib.mlem_forward(A, y, x3, e)
        rlib.mlem_back(A, e, c)
        rlib.mlem_update(x3, c, s, acc)
    # the scatter and gather paths sum the back projection in different orders
    assert torch.linalg.norm(x1 - x2) / torch.linalg.norm(x1) < 1e-5
    assert torch.linalg.norm(x1 - x3) / torch.linalg.norm(x1) < 1e-6


def test_reco_host_end_to_end(rlib, oracle, torch, small_full_matrix, small_measurement):
    A, _, _ = small_full_matrix
    g = cfg.SMALL
    y = small_measurement
    x, st = rlib.reco_host(g, y, 100, SEED, 20)
    s64, s = rlib.sensitivity(A)
    xr = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    rlib.Context(g, 0).mlem(A, torch.from_numpy(y).cuda(), s, xr, 20)
    xr = xr.cpu().numpy()
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < IMG_RTOL
    assert st["nnz"] == A.nnz and st["h2d_bytes"] >= y.nbytes and st["d2h_bytes"] == x.nbytes
    assert st["build_ms"] > 0 and st["iter_ms"] > 0


# ---------------------------------------------------------------- full-size properties

def test_full_size_matrix_properties(rlib, oracle, torch, ctx_full):
    """The whole 70^3 x 5.14M-channel matrix: structural invariants and a
    checksum of a row sample against the oracle (size-independent checks)."""
    g = cfg.FULL
    lst = np.arange(g.n_channels, dtype=np.int32)
    A = ctx_full.build(lst, 1000, SEED)
    rp = A.row_ptr
    assert int(rp[0]) == 0 and int(rp[-1]) == A.nnz
    assert bool((rp[1:] >= rp[:-1]).all())
    assert int(A.col.min()) >= 0 and int(A.col.max()) < g.n_voxels
    assert bool((A.val > 0).all())
    rng = np.random.Generator(np.random.PCG64(77))
    sample = np.sort(rng.choice(g.n_channels, 64, replace=False)).astype(np.int32)
    rp_o, col_o, val_o = oracle.sysmat(g, sample, 1000, SEED, method=1)
    rp_h = rp.cpu().numpy()
    for k, r in enumerate(sample):
        b, e = rp_h[r], rp_h[r + 1]
        cg = A.col[b:e].cpu().numpy()
        vg = A.val[b:e].cpu().numpy()
        assert np.array_equal(cg, col_o[rp_o[k]:rp_o[k + 1]])
        assert np.max(np.abs(vg - val_o[rp_o[k]:rp_o[k + 1]]) / val_o[rp_o[k]:rp_o[k + 1]]) <= VAL_RTOL
        assert np.all(np.diff(cg) > 0)
    # a checksum of checksums: row sums (A * ones), column sums (FP64
    # sensitivity) and the plain sum of all values agree
    total = 0.0
    chunk = 1 << 28
    for i in range(0, A.nnz, chunk):
        total += float(A.val[i:i + chunk].double().sum())
    row_sums = rlib.spmv(rlib.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, torch.ones(A.n, device="cuda"))
    assert abs(float(row_sums.double().sum()) - total) <= 1e-5 * total
    s64, s = rlib.sensitivity(A)
    assert abs(float(s64.sum()) - total) <= 1e-9 * total


def test_full_size_transpose_properties(rlib, torch, ctx_full):
    """The transpose of the whole 70^3 x 5.14M-channel matrix (3.7e9
    entries, both radix passes): the column pointers are the column counts
    of the rows, row positions ascend within every column, the values sum
    as the rows' do, the rows sampled by the test above (checked against
    the oracle there) sit entry by entry in their columns with the same
    bits, and the FP64 column sums through the transpose equal those through
    the rows (size-independent checks)."""
    g = cfg.FULL
    A = ctx_full.build(np.arange(g.n_channels, dtype=np.int32), 1000, SEED)
    s_rows, _ = rlib.sensitivity(A, use_transpose=False)
    A.transpose()
    m, n, nnz = A.m, A.n, A.nnz
    cp = A.col_ptr
    assert int(cp[0]) == 0 and int(cp[-1]) == nnz
    chunk = 1 << 28
    counts = torch.zeros(n, dtype=torch.int64, device="cuda")
    total = ttotal = 0.0
    starts = cp[1:-1]
    for i in range(0, nnz, chunk):
        j = min(i + chunk, nnz)
        counts += torch.bincount(A.col[i:j].long(), minlength=n)
        total += float(A.val[i:j].double().sum())
        ttotal += float(A.tval[i:j].double().sum())
        ri = A.row_idx[i:min(j + 1, nnz)]  # one entry of overlap with the next chunk
        assert int(ri.min()) >= 0 and int(ri.max()) < m
        # a position not above its predecessor may only open a column
        desc = torch.nonzero(ri[1:] <= ri[:-1]).squeeze(1) + (i + 1)
        assert bool(torch.isin(desc, starts).all())
    assert torch.equal(cp[1:] - cp[:-1], counts)
    assert abs(ttotal - total) <= 1e-9 * total
    rng = np.random.Generator(np.random.PCG64(77))
    sample = np.sort(rng.choice(g.n_channels, 64, replace=False))
    for r in sample[:32]:
        b, e = int(A.row_ptr[r]), int(A.row_ptr[r + 1])
        cols = A.col[b:e].long()
        lo, lens = cp[cols], cp[cols + 1] - cp[cols]
        seg = torch.repeat_interleave(torch.arange(cols.numel(), device="cuda"), lens)
        idx = torch.arange(int(lens.sum()), device="cuda") + torch.repeat_interleave(lo - (torch.cumsum(lens, 0) - lens),
                                                                                       lens)
        hit = torch.nonzero(A.row_idx[idx] == int(A.row_rank[r])).squeeze(1)
        assert torch.equal(seg[hit], torch.arange(cols.numel(), device="cuda"))  # once in each of its columns
        assert torch.equal(A.tval[idx[hit]].view(torch.int32), A.val[b:e].view(torch.int32))
    s_csc, _ = rlib.sensitivity(A)
    assert torch.equal(s_csc == 0, s_rows == 0)
    assert float(((s_csc - s_rows).abs() / s_rows.clamp_min(1e-300)).max()) <= 1e-10


def test_matrix_memory_is_released(rlib, torch, ctx_small):
    """Device memory of a matrix (and its transpose) is returned once the
    Matrix and its tensor views are dropped: to the library's block cache,
    which trim_memory empties."""
    lst = np.arange(0, 60000, dtype=np.int32)
    A = ctx_small.build(lst, 100, SEED)  # warms the context scratch
    del A
    torch.cuda.synchronize()
    rlib.trim_memory()
    free0 = torch.cuda.mem_get_info()[0]
    A = ctx_small.build(lst, 100, SEED)
    A.transpose()
    nbytes = A.nnz * 16
    col_view = A.col[:10]
    del A
    torch.cuda.synchronize()
    rlib.trim_memory()
    assert torch.cuda.mem_get_info()[0] < free0 - nbytes // 2  # the view keeps it alive
    del col_view
    torch.cuda.synchronize()
    rlib.trim_memory()
    assert torch.cuda.mem_get_info()[0] > free0 - nbytes // 4


def test_zslab_rows_both_sort_paths(rlib, oracle, ctx_full):
    """z-slab rows come out of the dense kernel in column order either by the
    counting sort over their windows' (x, y) box (at most 1024 keys at
    H = 4096) or by the bitonic sort (larger boxes): rows of both kinds,
    chosen with the host restatement of the windows, against the oracle."""
    from test_slab_windows import boxes, windows

    g = cfg.FULL
    per = g.n0z * g.n0y * g.n1z * g.n1y
    rng = np.random.default_rng(31)
    small_box, large_box = [], []
    # large boxes: a few % of the z-slab rows near 46-56 degrees, where the
    # rays drift most in x from slab to slab
    for a in list(range(23, 29)) * 10 + list(range(40, 50)):
        for cnl in (a * per + rng.integers(0, per, 6)).tolist():
            win = windows(g, *boxes(oracle, g, cnl)[:2])
            if win is None or win[0] != 2:
                continue
            rows = win[1]
            wu = max(r[1] - r[0] + 1 for r in rows)
            wv = max(r[3] - r[2] + 1 for r in rows)
            nkeys = (max(r[0] for r in rows) + wu - min(r[0] for r in rows)) * \
                    (max(r[2] for r in rows) + wv - min(r[2] for r in rows))
            (small_box if nkeys <= 1024 else large_box).append(cnl)
    assert len(small_box) >= 8 and len(large_box) >= 6, (len(small_box), len(large_box))
    lst = np.array(small_box[:24] + large_box[:16], np.int32)
    A = ctx_full.build(lst, 1000, SEED)
    assert_rows_equal(*A.to_numpy(), *oracle.sysmat(g, lst, 1000, SEED, method=1))
