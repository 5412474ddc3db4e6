"""The CPU oracle against the reference's golden vectors and known answers.

The oracle (oracle/oracle.cpp) restates the reference algorithm; these tests
pin it to arrays produced by the reference's own code (tests/golden, made by
tests/golden/make_golden.py from oracle/_ref) and to the known answers of the
reference's unit tests.
"""
import ctypes as C

import numpy as np
import pytest

from raptr_b200 import config as cfg


def test_philox_known_answers(oracle):
    # Random123 philox4x32-10 known-answer vectors.
    assert list(oracle.philox([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_uniforms_in_half_open_unit_interval(oracle):
    u = np.concatenate([oracle.ray_uniforms(1251, c, r) for c in (0, 7, 99) for r in range(200)])
    assert u.min() > 0.0 and u.max() <= 1.0
    assert abs(u.mean() - 0.5) < 0.02


# src/tests/MeasurementSetupTrafo2CartCoordUT.cu:42-52 setup, val_t = double.
UT = dict(pos0x=-3.5, pos1x=3.5, n0z=4, n0y=4, n1z=4, n1y=4, da=60.0, segx=1.0, segy=1.0, segz=1.0)


def _trafo_d(oracle, det, ida, idz, idy, dice):
    out = np.zeros(3)
    oracle.lib().ora_trafo_d(UT["pos0x"], UT["pos1x"], UT["n0z"], UT["n0y"], UT["n1z"], UT["n1y"], UT["da"],
                             UT["segx"], UT["segy"], UT["segz"], det, ida, idz, idy, np.asarray(dice, np.float64), out)
    return out


def _check_norot(det, idz, idy, dice):
    # CalcCheckCoordsNoRot (src/tests/MeasurementSetupTrafo2CartCoordUT.cu:91-137)
    pos = UT["pos0x"] if det == 0 else UT["pos1x"]
    ny = UT["n0y"] if det == 0 else UT["n1y"]
    nz = UT["n0z"] if det == 0 else UT["n1z"]
    return np.array([pos + (-0.5 + dice[0]) * UT["segx"], ((-0.5 * ny + idy) + dice[1]) * UT["segy"],
                     ((-0.5 * nz + idz) + dice[2]) * UT["segz"]])


@pytest.mark.parametrize("det", [0, 1])
@pytest.mark.parametrize("dice", [(0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0),
                                  (0.1, 0.1, 0.1)])
def test_trafo_unit_cases_no_rotation(oracle, det, dice):
    # test_MeasurementSetupTrafo2CartCoord_001..024: exact equality in double.
    got = _trafo_d(oracle, det, 0, 0, 0, dice)
    assert np.array_equal(got, _check_norot(det, 0, 0, dice))
    # the "screwed" fail cases: +1 on every coordinate must differ
    assert np.all(got != _check_norot(det, 0, 0, dice) + 1.0)


def test_trafo_unit_case_rotated(oracle):
    # test_MeasurementSetupTrafo2CartCoord_025: det0, pixel 00, rotation 1, corner 000.
    got = _trafo_d(oracle, 0, 1, 0, 0, (0.0, 0.0, 0.0))
    chk = _check_norot(0, 0, 0, (0.0, 0.0, 0.0))
    # Rotate (src/tests/MeasurementSetupTrafo2CartCoordUT.cu:309-320)
    s = np.float64(np.float32(np.sin(np.float32(np.pi / 180.0 * 1 * 60.0))))
    c = np.float64(np.float32(np.cos(np.float32(np.pi / 180.0 * 1 * 60.0))))
    oz, ox = chk[2], chk[0]
    want = np.array([s * oz + c * ox, chk[1], c * oz - s * ox])
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-6)


def test_trafo_matches_reference_float(oracle, golden):
    g = cfg.FULL
    for det in (0, 1):
        for i in range(golden["trafo_pts"].shape[0]):
            ida, idz, idy = (int(v) for v in golden["trafo_ids"][i])
            got = oracle.trafo_f(g, det, ida, idz, idy, golden["trafo_pts"][i])[0]
            assert np.array_equal(got.view(np.uint32), golden["trafo_out"][det, i].view(np.uint32))


def test_channel_index_bijection(oracle):
    # src/tests/test_MeasurementSetupLinIndex.cu:57-66 (sampled + ends).
    g = cfg.FULL
    rng = np.random.Generator(np.random.PCG64(3))
    for cnl in list(rng.integers(0, g.n_channels, 2000)) + [0, g.n_channels - 1]:
        ida, id0z, id0y, id1z, id1y = oracle.channel_split(g, int(cnl))
        assert oracle.lib().ora_channel_lin(C.byref(oracle.to_ogeom(g)), id0z, id0y, id1z, id1y, ida) == cnl
        assert 0 <= ida < g.na and 0 <= id0z < 13 and 0 <= id1y < 13


def test_voxel_index_bijection_and_layout(oracle):
    # src/tests/test_VoxelGridLinIndex.cu:57-64 and the density layout of
    # src/tests/test_H5DensityWriter.cpp:89 (x slowest, z fastest).
    g = cfg.epet_geometry(5, 0.001, 1, 1.0)
    g = cfg.Geometry(grid_o=(0.1, 0.2, 0.3), grid_d=(1.0, 2.0, 3.0), grid_n=(5, 6, 7), pos0x=-1, pos1x=1, na=1,
                     n0z=1, n0y=1, n1z=1, n1y=1, da=1.0, segx=1, segy=1, segz=1)
    for v in range(5 * 6 * 7):
        ix, iy, iz = oracle.voxel_split(g, v)
        assert ix * 6 * 7 + iy * 7 + iz == v
    assert list(oracle.voxel_split(g, 1 * 6 * 7 + 2 * 7 + 3)) == [1, 2, 3]


def test_reference_index_functors(oracle):
    if not oracle.ref_available():
        pytest.skip("reference harness not built here")
    g = cfg.FULL
    R = oracle.ref()
    gs = C.byref(oracle.to_ogeom(g))
    for cnl in (0, 1, 12345, 2570490, g.n_channels - 1):
        a = np.zeros(5, np.int32)
        R.ref_channel_split(gs, cnl, a)
        assert np.array_equal(a, oracle.channel_split(g, cnl))
    for v in (0, 1, 4899, 171500, g.n_voxels - 1):
        a = np.zeros(3, np.int32)
        R.ref_voxel_split(gs, v, a)
        assert np.array_equal(a, oracle.voxel_split(g, v))


def test_intersection_length_matches_reference(oracle, golden):
    for box, ray, want in zip(golden["il_boxes"], golden["il_rays"], golden["il_len"]):
        got = np.float32(oracle.intersection_length(box, ray))
        assert got.view(np.uint32) == np.float32(want).view(np.uint32)


@pytest.mark.parametrize("pruned", [False, True])
def test_workqueue_matches_reference_rows(oracle, golden, pruned):
    g = cfg.SMALL
    c, v, cur = oracle.workqueue(g, golden["small_list"], pruned=pruned)
    assert np.array_equal(c, golden["small_cnl"]) and np.array_equal(v, golden["small_vxl"])
    assert cur == (golden["small_list"].size, 0)


def test_workqueue_cursor_chunks_match_reference(oracle, golden):
    # Limited searches resume exactly where the reference's cursor stops.
    g = cfg.SMALL
    cur = (0, 0)
    k = 0
    for n, cnt, want_cur in zip(golden["wq_sizes"], golden["wq_counts"], golden["wq_cursors"]):
        c, v, cur = oracle.workqueue(g, golden["wq_list"], cursor=cur, max_out=int(n))
        assert c.size == cnt
        assert np.array_equal(c, golden["wq_cnl"][k:k + cnt]) and np.array_equal(v, golden["wq_vxl"][k:k + cnt])
        assert tuple(cur) == tuple(want_cur)
        k += cnt


def test_workqueue_prefix_property(oracle):
    # src/tests/test_getWorkqueue.cu:206-218: a limited search is a prefix of the full one.
    g = cfg.SMALL
    lst = np.array([5, 600, 142000], np.int32)
    c, v, _ = oracle.workqueue(g, lst)
    for n in (1, 17, 3000, c.size - 1):
        c2, v2, _ = oracle.workqueue(g, lst, max_out=n)
        assert np.array_equal(c2, c[:n]) and np.array_equal(v2, v[:n])


@pytest.mark.parametrize("which", ["small", "full"])
def test_sysmat_keep_zeros_matches_reference(oracle, golden, which):
    g = cfg.SMALL if which == "small" else cfg.FULL
    nrays = 100 if which == "small" else 64
    lst = golden[f"{which}_list"]
    for method in (0, 1):
        rp, col, val = oracle.sysmat(g, lst, nrays, 1251, method=method, keep_zeros=True)
        rows = np.repeat(lst, np.diff(rp))
        assert np.array_equal(rows, golden[f"{which}_cnl"])
        assert np.array_equal(col, golden[f"{which}_vxl"])
        assert np.array_equal(val.view(np.uint32), golden[f"{which}_val"].view(np.uint32))


def test_sysmat_zero_free_is_keep_zeros_without_zeros(oracle, golden):
    g = cfg.SMALL
    lst = golden["small_list"]
    rp, col, val = oracle.sysmat(g, lst, 100, 1251, method=1)
    nz = golden["small_val"] != 0
    assert np.array_equal(col, golden["small_vxl"][nz])
    assert np.array_equal(val.view(np.uint32), golden["small_val"][nz].view(np.uint32))
    assert np.array_equal(np.repeat(lst, np.diff(rp)), golden["small_cnl"][nz])


def test_walk_equals_slab_on_axis_parallel_rays(oracle):
    # Rays parallel to a plane family (equal start/end coordinate) leave that
    # axis unconstrained in the reference's masked min/max; both oracle
    # methods must agree on them exactly.
    g = cfg.SMALL
    lst = np.array([40000, 40001], np.int32)
    rays = oracle.rays(g, lst, 16, 5)
    rays[0, :, 4] = rays[0, :, 1]          # y equal
    rays[1, :8, 5] = rays[1, :8, 2]        # z equal
    a = oracle.sysmat(g, lst, 16, 0, rays_in=rays, method=0)
    b = oracle.sysmat(g, lst, 16, 0, rays_in=rays, method=1)
    assert all(np.array_equal(x.view(np.uint32) if x.dtype == np.float32 else x, y.view(np.uint32)
                              if y.dtype == np.float32 else y) for x, y in zip(a, b))


def test_coo_sort_and_csr_known_answers(oracle):
    # src/tests/test_cusparseWrapper.cu:40-48: rows {0,1,1,1,2,2,3,3,3} -> {0,1,4,6,9}
    rp = oracle.coo2csr(np.array([0, 1, 1, 1, 2, 2, 3, 3, 3], np.int32), 4)
    assert list(rp) == [0, 1, 4, 6, 9]
    # src/tests/test_convertCsr2Ecsr.cu:27-46: -> {0, 3, 3, 5}
    e = oracle.csr2ecsr(np.array([2, 4, 6], np.int32), np.array([0, 0, 0, 3, 3, 3, 3, 5], np.int64))
    assert list(e) == [0, 3, 3, 5]
    # src/tests/cooSortUT.cu:68-145 dense 2x2 shuffled case restored exactly
    val = np.array([3, 1, 0, 2], np.float32)
    row = np.array([1, 0, 0, 1], np.int32)
    col = np.array([1, 1, 0, 0], np.int32)
    oracle.lib().ora_coo_sort(val, row, col, 4)
    assert list(row) == [0, 0, 1, 1] and list(col) == [0, 1, 0, 1] and list(val) == [0, 1, 2, 3]
    # empty
    oracle.lib().ora_coo_sort(np.zeros(0, np.float32), np.zeros(0, np.int32), np.zeros(0, np.int32), 0)


def test_coo_sort_matches_reference(oracle):
    if not oracle.ref_available():
        pytest.skip("reference harness not built here")
    rng = np.random.Generator(np.random.PCG64(1234))
    n = 500
    lin = rng.choice(40 * 50, n, replace=False)
    row = (lin // 50).astype(np.int32)
    col = (lin % 50).astype(np.int32)
    val = rng.random(n).astype(np.float32)
    a = [val.copy(), row.copy(), col.copy()]
    b = [val.copy(), row.copy(), col.copy()]
    oracle.lib().ora_coo_sort(a[0], a[1], a[2], n)
    oracle.ref().ref_coo_sort(b[0], b[1], b[2], n)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_mlem_operations_known_answers(oracle, golden):
    # src/tests/test_mlemOperations.cu:59-109
    n = 10
    A = ((np.arange(n) + 1) ** 2).astype(np.float32)
    B = np.full(n, 10, np.float32)
    Cc = (np.arange(n) + 1).astype(np.float32)
    D = np.zeros(n, np.float32)
    oracle.lib().ora_divides(D, A, Cc, n)
    assert np.array_equal(D, golden["mlem_divides"]) and np.array_equal(D, np.arange(1, n + 1, dtype=np.float32))
    oracle.lib().ora_divides_multiplies(D, A, B, Cc, n)
    assert np.array_equal(D, golden["mlem_divmul"])
    assert oracle.lib().ora_sum(D, n) == golden["mlem_sum"][0] == 550.0
    oracle.lib().ora_scales(D, np.float32(1.0 / 550.0), n)
    assert np.array_equal(D, golden["mlem_scaled"])


def test_divides_multiplies_zero_divisor_rule(oracle):
    # dvs += (dvs == 0): a zero sensitivity divides by one.
    D = np.zeros(2, np.float32)
    oracle.lib().ora_divides_multiplies(D, np.array([2, 3], np.float32), np.array([5, 7], np.float32),
                                        np.array([0, 2], np.float32), 2)
    assert list(D) == [10.0, 10.5]


def test_walk_chords_sum_to_path_length_in_grid(oracle):
    # The chords of a ray partition its path through the grid: their sum is
    # the length of the segment inside the grid box (computed here in
    # double), and every chord is at most a voxel diagonal.
    g = cfg.FULL
    lo = np.array(g.grid_o, np.float64)
    hi = lo + np.array(g.grid_d, np.float64) * np.array(g.grid_n)
    rays = oracle.rays(g, np.array([100, 2570490, 4000000, 5140979], np.int32), 25, 9).reshape(-1, 6)
    diag = float(np.linalg.norm(np.array(g.grid_d, np.float64)))
    for r in rays.astype(np.float64):
        d = r[3:] - r[:3]
        t0 = (lo - r[:3]) / d
        t1 = (hi - r[:3]) / d
        a_in = np.max(np.minimum(t0, t1))
        a_out = np.min(np.maximum(t0, t1))
        want = max(a_out - a_in, 0.0) * np.linalg.norm(d)
        vox, L = oracle.walk_ray(g, r.astype(np.float32))
        assert abs(L.astype(np.float64).sum() - want) <= 1e-5 * want
        assert L.max() <= diag * (1 + 1e-5)
        assert np.all(np.diff(np.argsort(vox)) != 0)


def test_mlem_oracle_fp32_close_to_fp64(oracle):
    g = cfg.SMALL
    lst = np.arange(0, g.n_channels, 97, dtype=np.int32)
    rp, col, val = oracle.sysmat(g, lst, 20, 1, method=1)
    m, n = lst.size, g.n_voxels
    xt = cfg.phantom(g, rods=False)
    y = oracle.spmv(0, m, n, rp, col, val, xt) * 1000 + 1
    s = oracle.column_sums_f64(m, n, rp, col, val)
    s /= s.sum()
    x0 = np.full(n, 1.0 / n)
    x32 = oracle.mlem(m, n, rp, col, val, y.astype(np.float32), s.astype(np.float32), x0.astype(np.float32), 5)
    x64 = oracle.mlem(m, n, rp, col, val, y.astype(np.float64), s, x0, 5, dtype=np.float64)
    assert np.linalg.norm(x32 - x64) / np.linalg.norm(x64) < 1e-4
    assert abs(x32.sum() - 1.0) < 1e-5
