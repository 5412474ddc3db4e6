"""The C ABI library loads and exports every entry point include/raptr_b200.h
declares (no compute call: these run without a GPU)."""
import ctypes as C
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "raptr_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(raptr_[a-z0-9_]+)\s*\(", src)))


def test_header_parses():
    names = header_functions()
    assert "raptr_sm_build" in names and "raptr_mlem" in names and len(names) >= 25


def test_library_exports_every_declared_symbol(rlib):
    lib = C.CDLL(rlib.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_layer_binds_every_declared_symbol(rlib):
    assert set(header_functions()) <= set(rlib._SIGNATURES)


def test_abi_version_and_error_string(rlib):
    L = rlib.lib()
    assert L.raptr_abi_version() == 6
    assert isinstance(L.raptr_last_error(), bytes)


def test_invalid_geometry_rejected_without_gpu(rlib):
    # validation happens before any device call
    g = rlib.geom_struct(rlib.SMALL)
    g.grid_n[0] = 0
    h = C.c_void_p()
    st = rlib.lib().raptr_ctx_create(C.byref(g), 0, C.byref(h))
    assert st == 1 and b"grid_n" in rlib.lib().raptr_last_error()


def test_built_for_sm100a_only(rlib):
    # the build script targets sm_100a exclusively
    from raptr_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
