"""The C++ template API (include/raptr_b200.hpp), compiled as a reference
driver would compile it: host-side traits here, the reco loop on the GPU."""
import os
import subprocess

import numpy as np
import pytest

from raptr_b200 import config as cfg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
FLAGS = ["-O2", "-std=c++17", "-ffp-contract=off", f"-I{ROOT}/include", "-I/usr/local/cuda/include",
         f"-L{ROOT}/raptr_b200", "-lraptr_b200", f"-Wl,-rpath,{ROOT}/raptr_b200", "-L/usr/local/cuda/lib64",
         "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64"]


def compile_cpp(src, tmp_path):
    exe = str(tmp_path / os.path.basename(src).replace(".cpp", ""))
    r = subprocess.run(["/usr/bin/g++", os.path.join(CPP, src), "-o", exe] + FLAGS, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_host_traits(rlib, oracle, tmp_path):
    exe = compile_cpp("shim_host.cpp", tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    assert "failures 0" in lines
    assert sum(1 for l in lines if l.startswith("ok ")) == 24
    g = cfg.epet_geometry(70, 0.002, 180, 2.0)
    for l in lines:
        if not l.startswith("trafo_f"):
            continue
        f = l.split()
        k = int(f[1])
        got = np.array([float.fromhex(v) for v in f[2:]], np.float32)
        p = np.array([0.125 * k, 0.5, 1.0 - 0.1 * k], np.float32)
        w0 = oracle.trafo_f(g, 0, 17 * k, k, 12 - k, p)[0]
        w1 = oracle.trafo_f(g, 1, 17 * k, 12 - k, k, p)[0]
        assert np.array_equal(got.view(np.uint32), np.concatenate([w0, w1]).view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("keep_zeros", [False, True])
def test_shim_reco_loop_on_gpu(rlib, oracle, tmp_path, keep_zeros):
    exe = compile_cpp("shim_reco.cpp", tmp_path)
    out = tmp_path / "x.bin"
    r = subprocess.run([exe, str(out)] + (["keep"] if keep_zeros else []), capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    x = np.fromfile(out, np.float32)
    # the same loop on the oracle: rows of the listed channels, y = 1e4 * A x_true
    g = cfg.SMALL
    lst = np.arange(0, g.n_channels, 301, dtype=np.int32)
    rp, col, val = oracle.sysmat(g, lst, 100, 1251, method=1, keep_zeros=keep_zeros)
    # the entry count the shim added to *nnz_devi: every candidate with
    # RAPTR_SM_KEEP_ZEROS (the reference's structure), else the non-zeros
    assert f"rows {lst.size} nnz {int(rp[-1])}" in r.stdout
    xt = cfg.phantom(g, rods=False)
    y = (oracle.spmv(0, lst.size, g.n_voxels, rp, col, val, xt) * 1e4).astype(np.float32)
    s = oracle.column_sums_f64(lst.size, g.n_voxels, rp, col, val)
    s = (s / s.sum()).astype(np.float32)
    x0 = np.full(g.n_voxels, np.float32(1.0 / g.n_voxels), np.float32)
    want = oracle.mlem(lst.size, g.n_voxels, rp, col, val, y, s, x0, 5)
    assert np.linalg.norm(x - want) / np.linalg.norm(want) < 1e-4
