"""Edge cases of the transpose and the iteration on the GPU: empty rows and
columns, unsorted and repeated columns within rows, one and two radix
passes, empty matrices, lists that repeat a channel (natural row order),
zero iterations."""
import numpy as np
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def csc_reference(m, n, rp, col, val):
    rows = np.repeat(np.arange(m), np.diff(rp))
    o = np.argsort(col, kind="stable")
    cp = np.zeros(n + 1, np.int64)
    cp[1:] = np.cumsum(np.bincount(col, minlength=n))
    return cp, rows[o].astype(np.int32), val[o]


def random_csr(rng, m, n, density, sort_rows=True):
    rp = [0]
    cols, vals = [], []
    for r in range(m):
        k = rng.binomial(n, density) if r % 7 else 0  # every 7th row empty
        c = rng.choice(n, size=k, replace=False)
        if sort_rows:
            c = np.sort(c)
        cols.append(c)
        vals.append(rng.random(k).astype(np.float32))
        rp.append(rp[-1] + k)
    return (np.array(rp, np.int64), np.concatenate(cols).astype(np.int32) if cols else np.zeros(0, np.int32),
            np.concatenate(vals).astype(np.float32) if vals else np.zeros(0, np.float32))


# n = 700: one pass; 5000 and 300000: a 9-bit first digit; 800000: two 10-bit digits
@pytest.mark.parametrize("n,sort_rows",
                         [(700, True), (700, False), (5000, True), (5000, False), (300000, True), (800000, True)])
def test_transpose_general_csr(rlib, torch, n, sort_rows):
    rng = np.random.default_rng(n + sort_rows)
    m = 3000
    rp, col, val = random_csr(rng, m, n, min(0.05, 40.0 / n), sort_rows)
    cp_ref, ri_ref, tv_ref = csc_reference(m, n, rp, col, val)
    t = lambda a: torch.from_numpy(a).cuda()
    cp, ri, tv = rlib.csr_transpose(m, n, t(rp), t(col), t(val))
    assert np.array_equal(cp.cpu().numpy(), cp_ref)
    assert np.array_equal(ri.cpu().numpy(), ri_ref)
    assert np.array_equal(tv.cpu().numpy().view(np.uint32), tv_ref.view(np.uint32))
    # in a given order
    order = rng.permutation(m).astype(np.int32)
    rank = np.empty(m, np.int64)
    rank[order] = np.arange(m)
    cp2, pos, tv2 = rlib.csr_transpose_ordered(m, n, t(rp), t(col), t(val), t(order))
    pr = rank[np.repeat(np.arange(m), np.diff(rp))]
    o = np.lexsort((pr, col))
    assert np.array_equal(cp2.cpu().numpy(), cp_ref)
    assert np.array_equal(pos.cpu().numpy(), pr[o])
    assert np.array_equal(tv2.cpu().numpy().view(np.uint32), val[o].view(np.uint32))


def test_transpose_empty_matrices(rlib, torch):
    for m in (0, 5):
        rp = torch.zeros(m + 1, dtype=torch.int64, device="cuda")
        col = torch.zeros(0, dtype=torch.int32, device="cuda")
        val = torch.zeros(0, dtype=torch.float32, device="cuda")
        cp, ri, tv = rlib.csr_transpose(m, 10, rp, col, val)
        assert cp.cpu().tolist() == [0] * 11 and ri.numel() == 0


def test_transpose_rejects_bad_columns(rlib, torch):
    rp = torch.tensor([0, 2, 3], dtype=torch.int64, device="cuda")
    col = torch.tensor([1, 9, 0], dtype=torch.int32, device="cuda")  # 9 >= n
    val = torch.ones(3, device="cuda")
    with pytest.raises(RuntimeError):
        rlib.csr_transpose(2, 5, rp, col, val)


def test_repeated_channels_keep_natural_order(rlib, torch):
    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    lst = np.array([5, 900, 5, 41000, 900, 120000], np.int32)
    A = ctx.build(lst, 50, 1251)
    A.transpose()
    assert A.row_order is None  # the list repeats channels
    rp, col, val = A.to_numpy()
    cp_ref, ri_ref, tv_ref = csc_reference(A.m, A.n, rp, col, val)
    assert np.array_equal(A.row_idx.cpu().numpy(), ri_ref)
    # the gather iteration equals the scatter iteration on the same rows
    y = torch.tensor([10.0, 3.0, 0.0, 7.0, 1.0, 2.0], device="cuda")
    s = torch.from_numpy((np.bincount(col, weights=val, minlength=A.n) + 1e-3).astype(np.float32)).cuda()
    s /= s.sum()
    x1 = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    x2 = x1.clone()
    ctx.mlem(A, y, s, x1, 4, use_graph=False)
    acc = torch.zeros(1, dtype=torch.float64, device="cuda")
    c = torch.zeros(A.n, device="cuda")
    for _ in range(4):
        rlib.mlem_project(A, y, x2, c)
        rlib.mlem_update(x2, c, s, acc)
    assert torch.allclose(x1, x2, rtol=1e-5, atol=1e-9)


def test_zero_iterations_leave_the_image(rlib, torch):
    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    A = ctx.build(np.arange(100, dtype=np.int32), 20, 1251)
    A.transpose()
    y = torch.ones(A.m, device="cuda")
    s = torch.full((A.n,), 1.0 / A.n, device="cuda")
    x = torch.rand(A.n, device="cuda")
    x0 = x.clone()
    ctx.mlem(A, y, s, x, 0)
    assert torch.equal(x, x0)


def test_freed_blocks_are_reused_and_trimmed(rlib, torch):
    # Large blocks the library frees are kept for its next allocations;
    # a rebuild into them gives the same matrix, and trim_memory hands them
    # back to the driver.
    import gc

    g = cfg.FULL
    ctx = rlib.Context(g, 0)
    lst = np.arange(60000, dtype=np.int32)
    A = ctx.build(lst, 200, 1251)
    A.transpose()
    rp0, col0, val0 = A.to_numpy()
    assert col0.nbytes >= (64 << 20)
    del A
    gc.collect()
    torch.cuda.synchronize()
    B = ctx.build(lst, 200, 1251)
    B.transpose()
    rp1, col1, val1 = B.to_numpy()
    assert np.array_equal(rp0, rp1) and np.array_equal(col0, col1)
    assert np.allclose(val0, val1, rtol=1e-6, atol=0)
    del B
    gc.collect()
    torch.cuda.synchronize()
    free_kept = torch.cuda.mem_get_info()[0]
    rlib.trim_memory()
    free_trimmed = torch.cuda.mem_get_info()[0]
    assert free_trimmed - free_kept >= 2 * col0.nbytes


def test_rows_that_overflow_the_first_table_are_rebuilt(rlib, oracle, torch):
    # A 25 mm grid of 0.5 mm voxels with 64 rays per channel starts at the
    # smallest row table (2048 entries); a quarter of the rows hold more
    # voxels than that, in both of the build's chunks (85,683 rows, 65,536
    # per chunk), so the build drains its pipeline, rebuilds those chunks at
    # the next level and carries on.  Rows from both chunks against the
    # oracle.
    g = cfg.Geometry(grid_o=(-0.0125,) * 3, grid_d=(0.0005,) * 3, grid_n=(50,) * 3, pos0x=-0.240, pos1x=0.240,
                     na=3, n0z=13, n0y=13, n1z=13, n1y=13, da=30.0, segx=0.020, segy=0.004, segz=0.004)
    ctx = rlib.Context(g, 0)
    lst = np.arange(g.n_channels, dtype=np.int32)
    A = ctx.build(lst, 64, 1251)
    rp, col, val = A.to_numpy()
    lens = np.diff(rp)
    big = np.nonzero(lens > 2048)[0]
    assert big.size > 0 and big.min() < 65536 <= big.max()
    rng = np.random.default_rng(4)
    pick = np.unique(np.concatenate([rng.choice(big[big < 65536], 10), rng.choice(big[big >= 65536], 10),
                                     rng.choice(lst.size, 20)]))
    rp_o, col_o, val_o = oracle.sysmat(g, lst[pick], 64, 1251, method=1)
    for k, i in enumerate(pick):
        got_c = col[rp[i]:rp[i + 1]]
        got_v = val[rp[i]:rp[i + 1]]
        want_c = col_o[rp_o[k]:rp_o[k + 1]]
        want_v = val_o[rp_o[k]:rp_o[k + 1]].astype(np.float64)
        assert np.array_equal(got_c, want_c), f"row {i}"
        if want_v.size:
            assert np.max(np.abs(got_v - want_v) / want_v) <= 1e-5, f"row {i}"
