"""ctypes wrapper around the CPU oracle (liboracle.so) and the reference harness
(_ref/libraptr_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
the cpu_baseline leg of bench.py, as the checker.  The product package
(raptr_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libraptr_ref.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class OGeom(C.Structure):
    """Same layout as the oracle's OGeom and the library's raptr_geom."""

    _fields_ = [
        ("grid_o", C.c_float * 3),
        ("grid_d", C.c_float * 3),
        ("grid_n", C.c_int32 * 3),
        ("pos0x", C.c_float),
        ("pos1x", C.c_float),
        ("na", C.c_int32),
        ("n0z", C.c_int32),
        ("n0y", C.c_int32),
        ("n1z", C.c_int32),
        ("n1y", C.c_int32),
        ("da", C.c_float),
        ("segx", C.c_float),
        ("segy", C.c_float),
        ("segz", C.c_float),
    ]


def to_ogeom(g) -> OGeom:
    o = OGeom()
    for i in range(3):
        o.grid_o[i] = g.grid_o[i]
        o.grid_d[i] = g.grid_d[i]
        o.grid_n[i] = g.grid_n[i]
    for f in ("pos0x", "pos1x", "na", "n0z", "n0y", "n1z", "n1y", "da", "segx", "segy", "segz"):
        setattr(o, f, getattr(g, f))
    return o


def build(quiet: bool = True) -> None:
    """Compiles the oracle (and the reference harness where the reference
    sources are present) with oracle/Makefile."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        G = C.POINTER(OGeom)
        sig = {
            "ora_abi_version": (C.c_int, []),
            "ora_philox4x32_10": (None, [_u32p, _u32p, _u32p]),
            "ora_ray_uniforms": (None, [C.c_uint32, C.c_int64, C.c_int64, _f32p]),
            "ora_ray_uniforms_batch": (None, [C.c_uint32, _i32p, C.c_int64, C.c_int32, _f32p]),
            "ora_channel_split": (None, [G, C.c_int64, _i32p]),
            "ora_channel_lin": (C.c_int64, [G, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
            "ora_voxel_split": (None, [G, C.c_int64, _i32p]),
            "ora_angle_sincos": (None, [G, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
            "ora_trafo_f": (None, [G, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _f32p, _f32p, C.c_int64]),
            "ora_trafo_d": (None, [C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                   _f64p, _f64p]),
            "ora_candidate_test": (C.c_int, [G, C.c_int64, C.c_int64]),
            "ora_intersection_length": (C.c_float, [_f32p, _f32p]),
            "ora_rays": (None, [G, _i32p, C.c_int64, C.c_int32, C.c_uint32, _f32p]),
            "ora_walk_ray": (C.c_int64, [G, _f32p, _i32p, _f32p, C.c_int64]),
            "ora_workqueue": (C.c_int64, [G, _i32p, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int64,
                                          _i32p, _i32p, C.c_int]),
            "ora_candidate_counts": (None, [G, _i32p, C.c_int64, _i64p, C.c_int]),
            "ora_sysmat_build": (C.c_void_p, [G, _i32p, C.c_int64, C.c_int32, C.c_uint32, C.c_void_p, C.c_int, C.c_int,
                                              C.c_int]),
            "ora_csr_nnz": (C.c_int64, [C.c_void_p]),
            "ora_csr_copy": (None, [C.c_void_p, _i64p, _i32p, _f32p]),
            "ora_csr_free": (None, [C.c_void_p]),
            "ora_coo_sort": (None, [_f32p, _i32p, _i32p, C.c_int64]),
            "ora_coo2csr": (None, [_i32p, C.c_int64, C.c_int64, _i64p]),
            "ora_csr2ecsr": (None, [_i64p, _i32p, C.c_int64, _i64p, C.c_int64]),
            "ora_spmv_f32": (None, [C.c_int, C.c_int64, C.c_int64, _i64p, _i32p, _f32p, C.c_float, _f32p, C.c_float,
                                    _f32p]),
            "ora_spmv_f64": (None, [C.c_int, C.c_int64, C.c_int64, _i64p, _i32p, _f32p, C.c_double, _f64p, C.c_double,
                                    _f64p]),
            "ora_divides": (None, [_f32p, _f32p, _f32p, C.c_int64]),
            "ora_divides_multiplies": (None, [_f32p, _f32p, _f32p, _f32p, C.c_int64]),
            "ora_scales": (None, [_f32p, C.c_float, C.c_int64]),
            "ora_sum": (C.c_float, [_f32p, C.c_int64]),
            "ora_column_sums_f64": (None, [C.c_int64, C.c_int64, _i64p, _i32p, _f32p, _f64p]),
            "ora_mlem_f32": (None, [C.c_int64, C.c_int64, _i64p, _i32p, _f32p, _f32p, _f32p, _f32p, C.c_int32]),
            "ora_mlem_f64": (None, [C.c_int64, C.c_int64, _i64p, _i32p, _f32p, _f64p, _f64p, _f64p, C.c_int32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    """The reference's own code, instantiated on the host (oracle/_ref)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(REF_PATH)
        L = C.CDLL(REF_PATH)
        G = C.POINTER(OGeom)
        sig = {
            "ref_abi_version": (C.c_int, []),
            "ref_workqueue": (C.c_int64, [G, _i32p, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int32,
                                          _i32p, _i32p]),
            "ref_intersection_length": (C.c_float, [_f32p, _f32p]),
            "ref_trafo": (None, [G, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _f32p, _f32p]),
            "ref_channel_split": (None, [G, C.c_int32, _i32p]),
            "ref_channel_lin": (C.c_int32, [G, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
            "ref_voxel_split": (None, [G, C.c_int32, _i32p]),
            "ref_voxel_lin": (C.c_int32, [G, C.c_int32, C.c_int32, C.c_int32]),
            "ref_sysmat": (C.c_int64, [G, _i32p, C.c_int64, C.c_int32, _f32p, C.c_int64, _i32p, _i32p, _f32p]),
            "ref_get_chords": (C.c_int64, [_f32p, _f32p, _f32p, _i32p, C.c_int64, _f32p, _i32p]),
            "ref_coo_sort": (None, [_f32p, _i32p, _i32p, C.c_int32]),
            "ref_divides": (None, [_f32p, _f32p, _f32p, C.c_int32]),
            "ref_divides_multiplies": (None, [_f32p, _f32p, _f32p, _f32p, C.c_int32]),
            "ref_scales": (None, [_f32p, C.c_float, C.c_int32]),
            "ref_sum": (C.c_float, [_f32p, C.c_int32]),
            "ref_csr2ecsr": (None, [_i32p, _i32p, C.c_int32, _i32p, C.c_int32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _ref = L
    return _ref


# ---------------------------------------------------------------------------
# Convenience wrappers
# ---------------------------------------------------------------------------

def _g(g):
    return C.byref(to_ogeom(g))


def philox(ctr, key):
    out = np.zeros(4, np.uint32)
    lib().ora_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
    return out


def ray_uniforms(seed, cnl, ray):
    u = np.zeros(6, np.float32)
    lib().ora_ray_uniforms(seed, cnl, ray, u)
    return u


def ray_uniforms_batch(seed, cnl, nrays):
    cnl = np.ascontiguousarray(cnl, np.int32)
    out = np.zeros((cnl.size, nrays, 6), np.float32)
    lib().ora_ray_uniforms_batch(seed, cnl, cnl.size, nrays, out)
    return out


def channel_split(g, cnl):
    out = np.zeros(5, np.int32)
    lib().ora_channel_split(_g(g), cnl, out)
    return out


def voxel_split(g, v):
    out = np.zeros(3, np.int32)
    lib().ora_voxel_split(_g(g), v, out)
    return out


def angle_sincos(g, ida):
    s, c = C.c_float(), C.c_float()
    lib().ora_angle_sincos(_g(g), ida, C.byref(s), C.byref(c))
    return s.value, c.value


def sincos_table(g):
    t = np.zeros((g.na, 2), np.float32)
    for a in range(g.na):
        t[a] = angle_sincos(g, a)
    return t


def trafo_f(g, det, ida, idz, idy, pts):
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    out = np.zeros_like(pts)
    lib().ora_trafo_f(_g(g), det, ida, idz, idy, pts, out, pts.shape[0])
    return out


def candidate_test(g, cnl, vxl):
    return bool(lib().ora_candidate_test(_g(g), cnl, vxl))


def intersection_length(box, ray):
    return lib().ora_intersection_length(np.asarray(box, np.float32), np.asarray(ray, np.float32))


def rays(g, cnl, nrays, seed):
    cnl = np.ascontiguousarray(cnl, np.int32)
    out = np.zeros((cnl.size, nrays, 6), np.float32)
    lib().ora_rays(_g(g), cnl, cnl.size, nrays, seed, out)
    return out


def walk_ray(g, ray, cap=4096):
    v = np.zeros(cap, np.int32)
    L = np.zeros(cap, np.float32)
    n = lib().ora_walk_ray(_g(g), np.asarray(ray, np.float32), v, L, cap)
    assert n <= cap
    return v[:n], L[:n]


def workqueue(g, lst, cursor=(0, 0), max_out=1 << 62, pruned=True, cap=None):
    lst = np.ascontiguousarray(lst, np.int32)
    if cap is None:
        cap = int(min(max_out, lst.size * int(np.prod(g.grid_n))))
    out_c = np.zeros(max(cap, 1), np.int32)
    out_v = np.zeros(max(cap, 1), np.int32)
    cl, cv = C.c_int64(cursor[0]), C.c_int64(cursor[1])
    n = lib().ora_workqueue(_g(g), lst, lst.size, C.byref(cl), C.byref(cv), min(max_out, cap), out_c, out_v,
                            1 if pruned else 0)
    return out_c[:n].copy(), out_v[:n].copy(), (cl.value, cv.value)


def candidate_counts(g, lst, nthreads=0):
    lst = np.ascontiguousarray(lst, np.int32)
    out = np.zeros(lst.size, np.int64)
    lib().ora_candidate_counts(_g(g), lst, lst.size, out, nthreads)
    return out


def sysmat(g, lst, nrays, seed, rays_in=None, method=1, keep_zeros=False, nthreads=0):
    """Rows of the listed channels as CSR (row_ptr int64, col int32, val f32)."""
    lst = np.ascontiguousarray(lst, np.int32)
    rp_ = None
    if rays_in is not None:
        rays_in = np.ascontiguousarray(rays_in, np.float32)
        assert rays_in.size == lst.size * nrays * 6
        rp_ = rays_in.ctypes.data
    h = lib().ora_sysmat_build(_g(g), lst, lst.size, nrays, seed, rp_, method, 1 if keep_zeros else 0, nthreads)
    nnz = lib().ora_csr_nnz(h)
    rp = np.zeros(lst.size + 1, np.int64)
    col = np.zeros(max(nnz, 1), np.int32)
    val = np.zeros(max(nnz, 1), np.float32)
    lib().ora_csr_copy(h, rp, col, val)
    lib().ora_csr_free(h)
    return rp, col[:nnz], val[:nnz]


def coo2csr(rows, m):
    rows = np.ascontiguousarray(rows, np.int32)
    rp = np.zeros(m + 1, np.int64)
    lib().ora_coo2csr(rows, rows.size, m, rp)
    return rp


def csr2ecsr(yrow, csr):
    yrow = np.ascontiguousarray(yrow, np.int32)
    csr = np.ascontiguousarray(csr, np.int64)
    out = np.zeros(yrow.size + 1, np.int64)
    lib().ora_csr2ecsr(out, yrow, yrow.size, csr, csr.size - 1)
    return out


def spmv(op, m, n, rp, col, val, x, alpha=1.0, beta=0.0, y=None, dtype=np.float32):
    f = lib().ora_spmv_f32 if dtype == np.float32 else lib().ora_spmv_f64
    out_len = m if op == 0 else n
    y = np.zeros(out_len, dtype) if y is None else np.ascontiguousarray(y, dtype).copy()
    f(op, m, n, np.ascontiguousarray(rp, np.int64), np.ascontiguousarray(col, np.int32),
      np.ascontiguousarray(val, np.float32), alpha, np.ascontiguousarray(x, dtype), beta, y)
    return y


def column_sums_f64(m, n, rp, col, val):
    s = np.zeros(n, np.float64)
    lib().ora_column_sums_f64(m, n, np.ascontiguousarray(rp, np.int64), np.ascontiguousarray(col, np.int32),
                              np.ascontiguousarray(val, np.float32), s)
    return s


def mlem(m, n, rp, col, val, y, s, x0, niter, dtype=np.float32):
    x = np.ascontiguousarray(x0, dtype).copy()
    f = lib().ora_mlem_f32 if dtype == np.float32 else lib().ora_mlem_f64
    f(m, n, np.ascontiguousarray(rp, np.int64), np.ascontiguousarray(col, np.int32),
      np.ascontiguousarray(val, np.float32), np.ascontiguousarray(y, dtype), np.ascontiguousarray(s, dtype), x, niter)
    return x
