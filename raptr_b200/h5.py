"""HDF5 measurement and density files (the reference's formats) through the
library's libhdf5-free reader/writer (include/raptr_b200_h5.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib
from .config import Geometry

_SIGS = {
    "raptr_h5_last_error": (C.c_char_p, []),
    "raptr_h5_write_measurement": (C.c_int, [C.c_char_p, C.c_void_p, C.POINTER(C.c_int64)]),
    "raptr_h5_write_density": (C.c_int, [C.c_char_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_float),
                                         C.POINTER(C.c_float)]),
    "raptr_h5_dataset_info": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "raptr_h5_read_f32": (C.c_int, [C.c_char_p, C.c_char_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    "raptr_h5_read_density_grid": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_float),
                                             C.POINTER(C.c_float)]),
}


class H5Error(RuntimeError):
    pass


def _L():
    L = lib()
    for name, (res, args) in _SIGS.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    return L


def _check(st: int):
    if st != 0:
        raise H5Error(f"HDF5 status {st}: {_L().raptr_h5_last_error().decode()}")


def write_measurement(path: str, y, geom: Geometry):
    """Dataset "messung" (angles, z0, y0, z1, y1) of all channels."""
    y = np.ascontiguousarray(y, np.float32)
    if y.size != geom.n_channels:
        raise ValueError("one count per channel expected")
    dims = (C.c_int64 * 5)(geom.na, geom.n0z, geom.n0y, geom.n1z, geom.n1y)
    _check(_L().raptr_h5_write_measurement(path.encode(), y.ctypes.data, dims))


def write_density(path: str, x, geom: Geometry):
    """Dataset "density" (nx, ny, nz) with the grid attributes."""
    x = np.ascontiguousarray(x, np.float32)
    n = (C.c_int32 * 3)(*geom.grid_n)
    lo = (C.c_float * 3)(*geom.grid_o)
    hi = (C.c_float * 3)(*[np.float32(o) + np.float32(d) * np.float32(k)
                           for o, d, k in zip(geom.grid_o, geom.grid_d, geom.grid_n)])
    if x.size != int(np.prod(geom.grid_n)):
        raise ValueError("one value per voxel expected")
    _check(_L().raptr_h5_write_density(path.encode(), x.ctypes.data, n, lo, hi))


def dataset_shape(path: str, name: str):
    rank = C.c_int32(0)
    dims = (C.c_int64 * 8)()
    _check(_L().raptr_h5_dataset_info(path.encode(), name.encode(), C.byref(rank), dims))
    return tuple(int(dims[i]) for i in range(rank.value))


def read(path: str, name: str) -> np.ndarray:
    """A dataset of the root group as float32, in its shape."""
    shape = dataset_shape(path, name)
    out = np.empty(int(np.prod(shape)) if shape else 1, np.float32)
    cnt = C.c_int64(0)
    _check(_L().raptr_h5_read_f32(path.encode(), name.encode(), out.ctypes.data, out.size, C.byref(cnt)))
    return out.reshape(shape)


def read_measurement(path: str) -> np.ndarray:
    return read(path, "messung")


def read_density(path: str):
    """(density (nx, ny, nz), {"n": (..), "min": (..), "max": (..)})."""
    n = (C.c_int32 * 3)()
    lo = (C.c_float * 3)()
    hi = (C.c_float * 3)()
    _check(_L().raptr_h5_read_density_grid(path.encode(), n, lo, hi))
    return read(path, "density"), {"n": tuple(n), "min": tuple(lo), "max": tuple(hi)}
