"""The command-line drivers with the reference's argv (reco,
backprojection, pureSMCalculation): argument and file errors on the host;
on the GPU, their outputs equal the library's Python path on the same
files."""
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
def test_reco_backprojection_and_build_match_python(rlib, drivers, tmp_path):
    import torch

    g0 = cfg.SMALL
    nrays = 40
    # sensitivity of all channels and a measurement, as the library computes them
    ctx = rlib.Context(g0, 0)
    A_all = ctx.build(np.arange(g0.n_channels, dtype=np.int32), nrays, 1251)
    s64, s32 = rlib.sensitivity(A_all)
    sfile = str(tmp_path / "sens.h5")
    h5.write_density(sfile, s64.float().cpu().numpy(), g0)
    g = grid_geometry(sfile)
    ctx = rlib.Context(g, 0)
    A_all = ctx.build(np.arange(g.n_channels, dtype=np.int32), nrays, 1251)
    lam = rlib.spmv(rlib.OP_N, A_all.m, A_all.n, A_all.row_ptr, A_all.col, A_all.val,
                    torch.from_numpy(cfg.phantom(g, rods=False)).cuda()).cpu().numpy()
    y = cfg.poisson_measurement(lam, 1e5, 11)
    mfile = str(tmp_path / "meas.h5")
    h5.write_measurement(mfile, y, g)
    env = {"RAPTR_SETUP": SETUP, "RAPTR_GRID": "{},{},{},{},{},{},{},{},{}".format(*g.grid_n, *g.grid_o, *g.grid_d)}

    # reco: 3 iterations from a missing guess (all ones), outputs per iteration
    out = str(tmp_path / "out.h5")
    r = run(drivers["reco"], mfile, out, nrays, sfile, 3, str(tmp_path / "none.h5"), env=env)
    assert r.returncode == 0, r.stderr + r.stdout
    rows = np.nonzero(y)[0].astype(np.int32)
    A = ctx.build(rows, nrays, 1251)
    A.transpose()
    s = torch.from_numpy(h5.read_density(sfile)[0].ravel()).cuda()
    s = s / s.sum()
    x = torch.ones(g.n_voxels, device="cuda")
    yd = torch.from_numpy(y[rows]).cuda()
    for it in range(3):
        ctx.mlem(A, yd, s, x, 1, use_graph=False)
        d, grid = h5.read_density(str(tmp_path / f"{it}_out.h5"))
        assert grid["n"] == tuple(g.grid_n)
        want = x.cpu().numpy()
        assert np.linalg.norm(d.ravel() - want) / np.linalg.norm(want) < 1e-6

    # backprojection: normalised A^T y
    bout = str(tmp_path / "bp.h5")
    r = run(drivers["backprojection"], mfile, bout, nrays, env=env)
    assert r.returncode == 0, r.stderr
    bp = rlib.spmv(rlib.OP_T, A.m, A.n, A.row_ptr, A.col, A.val, yd).cpu().numpy()
    bp = bp / bp.sum()
    d, _ = h5.read_density(bout)
    assert np.linalg.norm(d.ravel() - bp) / np.linalg.norm(bp) < 1e-5

    # pureSMCalculation: the same number of entries
    r = run(drivers["pureSMCalculation"], mfile, nrays, env=env)
    assert r.returncode == 0, r.stderr
    assert f"entries {A.nnz}," in r.stdout
