"""The command-line drivers with the reference's argv (reco,
backprojection, pureSMCalculation): argument and file errors on the host;
on the GPU, their output files match the CPU oracle on the same
geometry, rays and measurement."""
import os
import subprocess

import numpy as np
import pytest

from raptr_b200 import config as cfg
from raptr_b200 import h5

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SETUP = "-0.240,0.240,36,0.020,0.004,0.004"  # the 5-angle ePET heads


@pytest.fixture(scope="module")
def drivers(rlib):
    from raptr_b200 import build

    return dict(zip(build.DRIVERS, build.build_drivers()))


def run(exe, *args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([exe, *map(str, args)], capture_output=True, text=True, env=e, timeout=600)


def test_usage_and_missing_files(drivers, tmp_path):
    r = run(drivers["reco"], "a", "b")
    assert r.returncode != 0 and "filename of density guess" in r.stderr
    r = run(drivers["backprojection"])
    assert r.returncode != 0 and "number of rays" in r.stderr
    r = run(drivers["pureSMCalculation"], str(tmp_path / "missing.h5"), 10)
    assert r.returncode != 0 and "cannot open" in r.stderr
    g = cfg.epet_geometry(8, 0.003, 1, 90.0)
    m = tmp_path / "m.h5"
    h5.write_measurement(str(m), np.ones(g.n_channels, np.float32), g)
    r = run(drivers["backprojection"], m, tmp_path / "o.h5", 10, env={"RAPTR_GRID": "1,2"})
    assert r.returncode != 0 and "RAPTR_GRID" in r.stderr


def grid_geometry(path):
    """The geometry the drivers derive: the grid from a density file's
    attributes (pitch = (max - min) / n in float), the heads of SETUP."""
    _, grid = h5.read_density(path)
    n = grid["n"]
    lo = np.array(grid["min"], np.float32)
    d = (np.array(grid["max"], np.float32) - lo) / np.array(n, np.float32)
    return cfg.Geometry(grid_o=tuple(float(v) for v in lo), grid_d=tuple(float(v) for v in d),
                        grid_n=tuple(int(v) for v in n), pos0x=-0.240, pos1x=0.240, na=5, n0z=13, n0y=13, n1z=13,
                        n1y=13, da=36.0, segx=0.020, segy=0.004, segz=0.004)


@pytest.mark.gpu
def test_reco_backprojection_and_build_match_the_oracle(rlib, oracle, drivers, tmp_path):
    """The drivers' files against the CPU oracle on the same geometry and
    rays: reco's density after every iteration ("<it>_<output>",
    src/tests/reco.cu:305-311) against the oracle's MLEM over the measured
    rows (src/tests/reco.cu:229-321), backprojection's normalised A^T y
    (src/tests/backprojection.cu:156-189) against the oracle's transposed
    CSRmv, and pureSMCalculation's entry count against the oracle's rows."""
    g0 = cfg.SMALL
    nrays = 40
    # the grid the drivers read from the sensitivity file's attributes
    sfile = str(tmp_path / "sens.h5")
    h5.write_density(sfile, np.ones(g0.n_voxels, np.float32), g0)
    g = grid_geometry(sfile)
    # a measurement of 6000 random channels, Poisson counts of the oracle's rows
    rng = np.random.default_rng(5)
    cand = np.sort(rng.choice(g.n_channels, 6000, replace=False)).astype(np.int32)
    rp_c, col_c, val_c = oracle.sysmat(g, cand, nrays, 1251, method=1)
    lam = oracle.spmv(0, cand.size, g.n_voxels, rp_c, col_c, val_c, cfg.phantom(g, rods=False).astype(np.float64),
                      dtype=np.float64)
    yc = cfg.poisson_measurement(lam, 2e5, 11)
    y = np.zeros(g.n_channels, np.float32)
    y[cand] = yc
    rows = np.nonzero(y)[0].astype(np.int32)
    rp, col, val = oracle.sysmat(g, rows, nrays, 1251, method=1)
    m, n = rows.size, g.n_voxels
    # sensitivity: FP64 column sums of the measured rows, written as the
    # file reco reads
    s64 = oracle.column_sums_f64(m, n, rp, col, val)
    h5.write_density(sfile, s64.astype(np.float32), g0)  # the same grid attributes as before
    assert grid_geometry(sfile) == g
    mfile = str(tmp_path / "meas.h5")
    h5.write_measurement(mfile, y, g)
    env = {"RAPTR_SETUP": SETUP, "RAPTR_GRID": "{},{},{},{},{},{},{},{},{}".format(*g.grid_n, *g.grid_o, *g.grid_d)}

    # reco: 3 iterations from a missing guess (all ones), one file per iteration
    out = str(tmp_path / "out.h5")
    r = run(drivers["reco"], mfile, out, nrays, sfile, 3, str(tmp_path / "none.h5"), env=env)
    assert r.returncode == 0, r.stderr + r.stdout
    sf = h5.read_density(sfile)[0].ravel()
    s = (sf / np.float32(sf.astype(np.float64).sum())).astype(np.float32)
    for it in range(3):
        want = oracle.mlem(m, n, rp, col, val, y[rows], s, np.ones(n, np.float32), it + 1)
        d, grid = h5.read_density(str(tmp_path / f"{it}_out.h5"))
        assert grid["n"] == tuple(g.grid_n)
        assert np.linalg.norm(d.ravel() - want) / np.linalg.norm(want) < 1e-4

    # backprojection: A^T y normalised to sum 1
    bout = str(tmp_path / "bp.h5")
    r = run(drivers["backprojection"], mfile, bout, nrays, env=env)
    assert r.returncode == 0, r.stderr
    bp = oracle.spmv(1, m, n, rp, col, val, y[rows].astype(np.float64), dtype=np.float64)
    bp = bp / bp.sum()
    d, _ = h5.read_density(bout)
    assert np.linalg.norm(d.ravel() - bp) / np.linalg.norm(bp) < 1e-5

    # pureSMCalculation: the oracle's number of entries
    r = run(drivers["pureSMCalculation"], mfile, nrays, env=env)
    assert r.returncode == 0, r.stderr
    assert f"entries {int(rp[-1])}," in r.stdout
