"""raptr_b200: the reconstruction hot path of raptr (candidate search, Monte
Carlo system matrix, CSR, MLEM) as hand-written sm_100a CUDA behind a C ABI
(include/raptr_b200.h, libraptr_b200.so).

This module is a thin ctypes layer over that library; PyTorch provides device
memory and streams.  There is no CPU fallback: if the library is missing or
no CUDA device is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

from .config import FINE, FULL, SMALL, WORKLOADS, Geometry, epet_geometry, phantom, poisson_measurement

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libraptr_b200.so")

RAPTR_OK = 0
RAPTR_ERR_CAPACITY = 3
OP_N = 0
OP_T = 1
SM_KEEP_ZEROS = 1

STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "CAPACITY", 4: "OVERFLOW", 5: "NOMEM", 6: "UNSUPPORTED"}


class RaptrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"raptr status {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class raptr_geom(C.Structure):
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


class raptr_mlem_opts(C.Structure):
    _fields_ = [("use_graph", C.c_int32), ("h_loglik", C.POINTER(C.c_double)), ("h_kernel_ms", C.POINTER(C.c_float)),
                ("d_row_rank", C.c_void_p)]


class raptr_server_opts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("max_frames", C.c_int32), ("keep_fp32", C.c_int32)]


class raptr_request_stats(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("run_ms", C.c_double), ("total_ms", C.c_double),
                ("iterations", C.c_int32), ("frames_max", C.c_int32), ("cold_build", C.c_int32)]


class raptr_server_stats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("submitted", "completed", "iterations", "batch_steps", "builds", "evictions",
                                         "resident_matrices", "resident_bytes", "queued", "running")]


class raptr_stream_stats(C.Structure):
    _fields_ = [("resident_rows", C.c_int64), ("resident_entries", C.c_int64), ("streamed_rows", C.c_int64),
                ("level", C.c_int32), ("first_iter_ms", C.c_double), ("iter_ms", C.c_double)]


class raptr_reco_stats(C.Structure):
    _fields_ = [
        ("build_ms", C.c_double),
        ("sens_ms", C.c_double),
        ("iter_ms", C.c_double),
        ("total_ms", C.c_double),
        ("nnz", C.c_int64),
        ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64),
        ("transpose_ms", C.c_double),
        ("inputs_ms", C.c_double),
        ("output_ms", C.c_double),
        ("setup_ms", C.c_double),
        ("release_ms", C.c_double),
        ("wall_ms", C.c_double),
        ("streamed_rows", C.c_int64),
    ]


def geom_struct(g: Geometry) -> raptr_geom:
    s = raptr_geom()
    for i in range(3):
        s.grid_o[i] = g.grid_o[i]
        s.grid_d[i] = g.grid_d[i]
        s.grid_n[i] = g.grid_n[i]
    for f in ("pos0x", "pos1x", "na", "n0z", "n0y", "n1z", "n1y", "da", "segx", "segy", "segz"):
        setattr(s, f, getattr(g, f))
    return s


_lib = None
VP = C.c_void_p
I64 = C.c_int64
I32 = C.c_int32
P64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes); every entry point of include/raptr_b200.h
_SIGNATURES = {
    "raptr_abi_version": (C.c_int, []),
    "raptr_last_error": (C.c_char_p, []),
    "raptr_kernel_launches": (I64, []),
    "raptr_trim_memory": (I32, [I32]),
    "raptr_ctx_create": (C.c_int, [C.POINTER(raptr_geom), C.c_int, C.POINTER(VP)]),
    "raptr_ctx_destroy": (C.c_int, [VP]),
    "raptr_ctx_num_channels": (I64, [VP]),
    "raptr_ctx_num_voxels": (I64, [VP]),
    "raptr_workqueue": (C.c_int, [VP, VP, I64, P64, P64, I64, VP, VP, P64, VP]),
    "raptr_candidate_counts": (C.c_int, [VP, VP, I64, VP, VP]),
    "raptr_rays": (C.c_int, [VP, VP, I64, I32, C.c_uint32, VP, VP]),
    "raptr_sm_build": (C.c_int, [VP, VP, I64, I32, C.c_uint32, VP, I32, I64, VP, VP, VP, P64, VP]),
    "raptr_sm_build_alloc": (C.c_int, [VP, VP, I64, I32, C.c_uint32, VP, I32, C.POINTER(VP), VP]),
    "raptr_matrix_info": (C.c_int, [VP, P64, P64, P64, C.POINTER(VP), C.POINTER(VP), C.POINTER(VP)]),
    "raptr_matrix_destroy": (C.c_int, [VP]),
    "raptr_coo2csr": (C.c_int, [VP, I64, I64, VP, VP]),
    "raptr_csr2ecsr": (C.c_int, [VP, VP, I64, VP, I64, VP]),
    "raptr_spmv": (C.c_int, [I32, I64, I64, VP, VP, VP, C.c_float, VP, C.c_float, VP, VP]),
    "raptr_divides": (C.c_int, [VP, VP, VP, I64, VP]),
    "raptr_divides_multiplies": (C.c_int, [VP, VP, VP, VP, I64, VP]),
    "raptr_scales": (C.c_int, [VP, C.c_float, I64, VP]),
    "raptr_sum": (C.c_int, [VP, I64, C.POINTER(C.c_double), VP]),
    "raptr_sensitivity": (C.c_int, [I64, I64, VP, VP, VP, VP, VP, VP]),
    "raptr_mlem_project": (C.c_int, [I64, VP, VP, VP, VP, VP, VP, VP, VP]),
    "raptr_mlem_update": (C.c_int, [I64, VP, VP, VP, VP, VP]),
    "raptr_mlem": (C.c_int, [VP, I64, I64, VP, VP, VP, VP, VP, VP, VP, VP, VP, I32, C.POINTER(raptr_mlem_opts),
                             VP]),
    "raptr_mlem_forward": (C.c_int, [I64, VP, VP, VP, VP, VP, VP, VP, VP]),
    "raptr_mlem_forward_ordered": (C.c_int, [I64, VP, VP, VP, VP, VP, VP, VP, VP, VP]),
    "raptr_mlem_back": (C.c_int, [I64, VP, VP, VP, VP, VP, VP]),
    "raptr_matrix_transpose": (C.c_int, [VP, VP]),
    "raptr_matrix_csc_info": (C.c_int, [VP, C.POINTER(VP), C.POINTER(VP), C.POINTER(VP)]),
    "raptr_matrix_row_order": (C.c_int, [VP, C.POINTER(VP), C.POINTER(VP)]),
    "raptr_matrix_half": (C.c_int, [VP, VP]),
    "raptr_matrix_half_info": (C.c_int, [VP, C.POINTER(VP), C.POINTER(VP), C.POINTER(VP), C.POINTER(VP)]),
    "raptr_sensitivity_half": (C.c_int, [I64, VP, VP, VP, VP, VP, VP, VP]),
    "raptr_sensitivity_csc": (C.c_int, [I64, VP, VP, VP, VP, VP]),
    "raptr_mlem_half": (C.c_int, [VP, I64, I64, VP, VP, VP, VP, VP, VP, VP, VP, VP, VP, I32,
                                  C.POINTER(raptr_mlem_opts), VP]),
    "raptr_pack_half": (C.c_int, [I64, VP, VP, VP, VP, VP, VP, I64, C.POINTER(I64), VP]),
    "raptr_matrix_packed": (C.c_int, [VP, VP]),
    "raptr_matrix_packed_info": (C.c_int, [VP] + [C.POINTER(VP)] * 6),
    "raptr_mlem_packed": (C.c_int, [VP, I64, I64, VP, VP, VP, VP, VP, VP, VP, VP, VP, VP, I32,
                                    C.POINTER(raptr_mlem_opts), VP]),
    "raptr_mlem_f64": (C.c_int, [VP, I64, I64, VP, VP, VP, VP, VP, VP, VP, VP, VP, VP, I32, VP, VP]),
    "raptr_mlem_batch": (C.c_int, [VP, I64, I64, I32, I32, VP, VP, VP, VP, VP, VP, VP, VP, VP, VP, VP, I32, I32,
                                   C.POINTER(raptr_mlem_opts), VP]),
    "raptr_mlem_batch_autotune": (C.c_int, [VP, I64, I64, I32, I32, VP, VP, VP, VP, VP, VP, VP, VP, VP, VP, VP,
                                            C.POINTER(C.c_int32), C.POINTER(C.c_float), VP]),
    "raptr_csr_transpose": (C.c_int, [I64, I64, VP, VP, VP, VP, VP, VP, VP]),
    "raptr_csr_transpose_ordered": (C.c_int, [I64, I64, VP, VP, VP, VP, VP, VP, VP, VP]),
    "raptr_mlem_noalloc": (C.c_int, [I64, I64, VP, VP, VP, VP, VP, VP, I32, VP]),
    "raptr_mlem_stream": (C.c_int, [VP, VP, I64, I32, C.c_uint32, VP, VP, VP, VP, I32, I64,
                                    C.POINTER(raptr_stream_stats), VP]),
    "raptr_row_ptr_narrow": (C.c_int, [VP, I64, VP, VP]),
    "raptr_row_ptr_widen": (C.c_int, [VP, I64, VP, VP]),
    "raptr_reco_host": (C.c_int, [C.POINTER(raptr_geom), C.c_int, VP, I32, C.c_uint32, I32, VP, VP, VP,
                                  C.POINTER(raptr_reco_stats)]),
    "raptr_matrix_drop_f32": (C.c_int, [VP]),
    "raptr_matrix_bytes": (C.c_int, [VP, C.POINTER(C.c_int64)]),
    "raptr_server_create": (C.c_int, [I32, C.POINTER(raptr_server_opts), C.POINTER(VP)]),
    "raptr_server_destroy": (C.c_int, [VP]),
    "raptr_server_submit": (C.c_int, [VP, C.POINTER(raptr_geom), I32, C.c_uint32, VP, I32, C.POINTER(C.c_int64)]),
    "raptr_server_wait": (C.c_int, [VP, C.c_int64, VP, I32, C.POINTER(raptr_request_stats)]),
    "raptr_server_get_stats": (C.c_int, [VP, C.POINTER(raptr_server_stats)]),
}


def lib():
    """Loads libraptr_b200.so (built in-tree by raptr_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python -m raptr_b200.build` (there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status != RAPTR_OK:
        raise RaptrError(status, lib().raptr_last_error().decode())


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("raptr_b200 needs a CUDA device (sm_100a); none is available")
    return torch


def _ptr(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


class _MatrixHandle:
    """Owns a raptr_matrix*; destroys it when the last reference goes (the
    Matrix object and every tensor view hold one)."""

    def __init__(self, handle: int):
        self.h = VP(handle)

    def __del__(self):
        if self.h.value and _lib is not None:
            _lib.raptr_matrix_destroy(self.h)
            self.h = VP(0)


class _DeviceArray:
    """Zero-copy __cuda_array_interface__ view of library-owned memory; keeps
    the owning handle alive (and nothing else, so no reference cycle)."""

    def __init__(self, ptr: int, shape, typestr: str, owner: _MatrixHandle):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}
        self._owner = owner


class Matrix:
    """System matrix rows held by the library (CSR: int64 row_ptr, int32 col,
    float32 val), resident in device memory.  The device memory is released
    when the Matrix and all tensor views of it are gone."""

    def __init__(self, handle: int, device: int):
        self._owner = _MatrixHandle(handle)
        self._h = self._owner.h
        self.device = device
        m, n, nnz = C.c_int64(), C.c_int64(), C.c_int64()
        rp, col, val = VP(), VP(), VP()
        _check(lib().raptr_matrix_info(self._h, C.byref(m), C.byref(n), C.byref(nnz), C.byref(rp), C.byref(col),
                                       C.byref(val)))
        self.m, self.n, self.nnz = m.value, n.value, nnz.value
        torch = _torch()
        dev = torch.device("cuda", device)
        own = self._owner
        self.row_ptr = torch.as_tensor(_DeviceArray(rp.value, (self.m + 1,), "<i8", own), device=dev)
        if self.nnz > 0:
            self.col = torch.as_tensor(_DeviceArray(col.value, (self.nnz,), "<i4", own), device=dev)
            self.val = torch.as_tensor(_DeviceArray(val.value, (self.nnz,), "<f4", own), device=dev)
        else:
            self.col = torch.zeros(0, dtype=torch.int32, device=dev)
            self.val = torch.zeros(0, dtype=torch.float32, device=dev)

    @property
    def has_transpose(self) -> bool:
        return self.col_ptr is not None

    col_ptr = None
    # back-projection order of the rows (row_idx of the transpose holds
    # positions k, row = row_order[k]); None for the natural order
    row_order = None
    row_rank = None
    row_idx = None
    tval = None

    def transpose(self, stream=None) -> "Matrix":
        """Builds the resident CSC copy used by the gather back projection."""
        _check(lib().raptr_matrix_transpose(self._h, _stream(stream)))
        cp, ri, tv = VP(), VP(), VP()
        _check(lib().raptr_matrix_csc_info(self._h, C.byref(cp), C.byref(ri), C.byref(tv)))
        torch = _torch()
        dev = torch.device("cuda", self.device)
        own = self._owner
        self.col_ptr = torch.as_tensor(_DeviceArray(cp.value, (self.n + 1,), "<i8", own), device=dev)
        if self.nnz > 0:
            self.row_idx = torch.as_tensor(_DeviceArray(ri.value, (self.nnz,), "<i4", own), device=dev)
            self.tval = torch.as_tensor(_DeviceArray(tv.value, (self.nnz,), "<f4", own), device=dev)
        else:
            self.row_idx = torch.zeros(0, dtype=torch.int32, device=dev)
            self.tval = torch.zeros(0, dtype=torch.float32, device=dev)
        order, rank = VP(), VP()
        _check(lib().raptr_matrix_row_order(self._h, C.byref(order), C.byref(rank)))
        if order.value and self.m > 0:
            self.row_order = torch.as_tensor(_DeviceArray(order.value, (self.m,), "<i4", own), device=dev)
            self.row_rank = torch.as_tensor(_DeviceArray(rank.value, (self.m,), "<i4", own), device=dev)
        return self

    # FP16 form (to_half): h values in CSR and transpose order, row scales
    hval = None
    rscale = None
    htval = None
    pscale = None

    def to_half(self, stream=None) -> "Matrix":
        """Builds the FP16 copy (a_ij ~= rscale_i * h_ij) beside the FP32
        matrix; transposes first if needed."""
        if not self.has_transpose:
            self.transpose(stream)
        _check(lib().raptr_matrix_half(self._h, _stream(stream)))
        hv, rs, ht, ps = VP(), VP(), VP(), VP()
        _check(lib().raptr_matrix_half_info(self._h, C.byref(hv), C.byref(rs), C.byref(ht), C.byref(ps)))
        torch = _torch()
        dev = torch.device("cuda", self.device)
        own = self._owner
        nz, mm = max(self.nnz, 1), max(self.m, 1)
        self.hval = torch.as_tensor(_DeviceArray(hv.value, (nz,), "<f2", own), device=dev)[:self.nnz]
        self.htval = torch.as_tensor(_DeviceArray(ht.value, (nz,), "<f2", own), device=dev)[:self.nnz]
        self.rscale = torch.as_tensor(_DeviceArray(rs.value, (mm,), "<f4", own), device=dev)[:self.m]
        self.pscale = torch.as_tensor(_DeviceArray(ps.value, (mm,), "<f4", own), device=dev)[:self.m]
        return self

    # delta-coded FP16 form (to_packed): rows and transpose columns as runs
    # of words (h << 16) | index step
    pseg = None
    panchor = None
    pword = None
    tseg = None
    tanchor = None
    tword = None

    def to_packed(self, stream=None) -> "Matrix":
        """Builds the delta-coded copy of the FP16 form (raptr_matrix_packed);
        builds the FP16 form first if needed."""
        if self.hval is None:
            self.to_half(stream)
        _check(lib().raptr_matrix_packed(self._h, _stream(stream)))
        p = [VP() for _ in range(6)]
        _check(lib().raptr_matrix_packed_info(self._h, *[C.byref(v) for v in p]))
        torch = _torch()
        dev = torch.device("cuda", self.device)
        own = self._owner
        self.pseg = torch.as_tensor(_DeviceArray(p[0].value, (self.m + 1,), "<i8", own), device=dev)
        self.tseg = torch.as_tensor(_DeviceArray(p[3].value, (self.n + 1,), "<i8", own), device=dev)
        nw, ntw = packed_words(self.pseg, self.m), packed_words(self.tseg, self.n)
        self.panchor = torch.as_tensor(_DeviceArray(p[1].value, (max(self.m, 1),), "<i4", own), device=dev)
        self.pword = torch.as_tensor(_DeviceArray(p[2].value, (max(nw, 4),), "<i4", own), device=dev)[:nw]
        self.tanchor = torch.as_tensor(_DeviceArray(p[4].value, (max(self.n, 1),), "<i4", own), device=dev)
        self.tword = torch.as_tensor(_DeviceArray(p[5].value, (max(ntw, 4),), "<i4", own), device=dev)[:ntw]
        return self

    def to_numpy(self):
        return self.row_ptr.cpu().numpy(), self.col.cpu().numpy(), self.val.cpu().numpy()


class Context:
    """Per-geometry device context (raptr_ctx)."""

    def __init__(self, geom: Geometry, device: int = 0):
        self.geom = geom
        self.device = device
        self._gs = geom_struct(geom)
        h = VP()
        _check(lib().raptr_ctx_create(C.byref(self._gs), device, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.raptr_ctx_destroy(h)
            self._h = VP(0)

    @property
    def n_channels(self) -> int:
        return lib().raptr_ctx_num_channels(self._h)

    @property
    def n_voxels(self) -> int:
        return lib().raptr_ctx_num_voxels(self._h)

    def _dev(self):
        torch = _torch()
        return torch.device("cuda", self.device)

    def _list(self, cnl):
        torch = _torch()
        t = torch.as_tensor(cnl, dtype=torch.int32, device=self._dev())
        return t.contiguous()

    # -- candidate search ----------------------------------------------------
    def workqueue(self, cnl, cursor: Tuple[int, int] = (0, 0), max_out: int = 1 << 20, stream=None):
        """getWorkqueue: (cnl, vxl) candidates in scan order from `cursor`,
        at most max_out; returns (cnl, vxl, new_cursor)."""
        torch = _torch()
        lst = self._list(cnl)
        oc = torch.empty(max(max_out, 1), dtype=torch.int32, device=self._dev())
        ov = torch.empty(max(max_out, 1), dtype=torch.int32, device=self._dev())
        li, vi, nf = C.c_int64(cursor[0]), C.c_int64(cursor[1]), C.c_int64()
        _check(lib().raptr_workqueue(self._h, _ptr(lst), lst.numel(), C.byref(li), C.byref(vi), max_out, _ptr(oc),
                                     _ptr(ov), C.byref(nf), _stream(stream)))
        n = nf.value
        return oc[:n], ov[:n], (li.value, vi.value)

    def candidate_counts(self, cnl, stream=None):
        torch = _torch()
        lst = self._list(cnl)
        out = torch.empty(lst.numel(), dtype=torch.int64, device=self._dev())
        _check(lib().raptr_candidate_counts(self._h, _ptr(lst), lst.numel(), _ptr(out), _stream(stream)))
        return out

    # -- rays and matrix -------------------------------------------------------
    def rays(self, cnl, nrays: int, seed: int, stream=None):
        torch = _torch()
        lst = self._list(cnl)
        out = torch.empty((lst.numel(), nrays, 6), dtype=torch.float32, device=self._dev())
        _check(lib().raptr_rays(self._h, _ptr(lst), lst.numel(), nrays, seed, _ptr(out), _stream(stream)))
        return out

    def build(self, cnl, nrays: int, seed: int, rays=None, keep_zeros: bool = False, stream=None) -> Matrix:
        """systemMatrixCalculation: rows for the listed channels, resident."""
        lst = self._list(cnl)
        rp = None
        if rays is not None:
            rays = rays.to(device=self._dev(), dtype=_torch().float32).contiguous()
            assert rays.numel() == lst.numel() * nrays * 6
            rp = _ptr(rays)
        h = VP()
        _check(lib().raptr_sm_build_alloc(self._h, _ptr(lst), lst.numel(), nrays, seed, rp,
                                          SM_KEEP_ZEROS if keep_zeros else 0, C.byref(h), _stream(stream)))
        return Matrix(h.value, self.device)

    def build_into(self, cnl, nrays: int, seed: int, row_ptr, col, val, rays=None, keep_zeros=False, stream=None):
        """raptr_sm_build into caller tensors; returns (status, nnz)."""
        lst = self._list(cnl)
        nnz = C.c_int64()
        st = lib().raptr_sm_build(self._h, _ptr(lst), lst.numel(), nrays, seed, _ptr(rays),
                                  SM_KEEP_ZEROS if keep_zeros else 0, 0 if col is None else col.numel(), _ptr(row_ptr),
                                  _ptr(col), _ptr(val), C.byref(nnz), _stream(stream))
        if st not in (RAPTR_OK, RAPTR_ERR_CAPACITY):
            _check(st)
        return st, nnz.value

    def mlem(self, A: Matrix, y, s, x, niter: int, use_graph: bool = True, loglik: bool = False,
             kernel_times: bool = False, stream=None):
        """MLEM iterations in place on x.  Returns the per-iteration
        log-likelihood (loglik) and/or the (n_iter, 2) device times in ms of
        the two passes of each iteration (kernel_times), else None."""
        ll = (C.c_double * max(niter, 1))() if loglik else None
        kt = (C.c_float * max(2 * niter, 1))() if kernel_times else None
        opts = raptr_mlem_opts(1 if use_graph else 0, C.cast(ll, C.POINTER(C.c_double)) if loglik else None,
                               C.cast(kt, C.POINTER(C.c_float)) if kernel_times else None,
                               _ptr(A.row_rank) if A.has_transpose else None)
        _check(lib().raptr_mlem(self._h, A.m, A.n, _ptr(A.row_ptr), _ptr(A.col), _ptr(A.val), _ptr(A.col_ptr),
                                _ptr(A.row_idx), _ptr(A.tval), _ptr(y), _ptr(s), _ptr(x), niter, C.byref(opts),
                                _stream(stream)))
        out = []
        if loglik:
            out.append(np.array(ll[:niter]))
        if kernel_times:
            out.append(np.array(kt[:2 * niter], np.float64).reshape(niter, 2))
        return None if not out else (out[0] if len(out) == 1 else tuple(out))


    def mlem_stream(self, cnl, nrays: int, seed: int, y, s, x, niter: int, resident_bytes: int, s_out=None,
                    stream=None) -> dict:
        """MLEM over the rows of the listed channels without storing the
        whole matrix: the leading rows that fit resident_bytes are kept after
        the first iteration, the others are rebuilt in every iteration
        (raptr_mlem_stream).  y: counts of the listed channels; s: the
        normalised sensitivity or None (computed; written to s_out when
        given); x updated in place.  Returns the call's statistics."""
        lst = self._list(cnl)
        st = raptr_stream_stats()
        _check(lib().raptr_mlem_stream(self._h, _ptr(lst), lst.numel(), nrays, seed, _ptr(y), _ptr(s), _ptr(s_out),
                                       _ptr(x), niter, int(resident_bytes), C.byref(st), _stream(stream)))
        return {k: getattr(st, k) for k, _ in raptr_stream_stats._fields_}

    def mlem_half(self, A: Matrix, y, s, x, niter: int, use_graph: bool = True, loglik: bool = False,
                  kernel_times: bool = False, stream=None):
        """MLEM iterations with A's FP16 copy (A.to_half()); as mlem()."""
        assert A.hval is not None, "call A.to_half() first"
        ll = (C.c_double * max(niter, 1))() if loglik else None
        kt = (C.c_float * max(2 * niter, 1))() if kernel_times else None
        opts = raptr_mlem_opts(1 if use_graph else 0, C.cast(ll, C.POINTER(C.c_double)) if loglik else None,
                               C.cast(kt, C.POINTER(C.c_float)) if kernel_times else None, _ptr(A.row_rank))
        _check(lib().raptr_mlem_half(self._h, A.m, A.n, _ptr(A.row_ptr), _ptr(A.col), _ptr(A.hval),
                                     _ptr(A.rscale), _ptr(A.col_ptr), _ptr(A.row_idx), _ptr(A.htval), _ptr(y),
                                     _ptr(s), _ptr(x), niter, C.byref(opts), _stream(stream)))
        out = []
        if loglik:
            out.append(np.array(ll[:niter]))
        if kernel_times:
            out.append(np.array(kt[:2 * niter], np.float64).reshape(niter, 2))
        return None if not out else (out[0] if len(out) == 1 else tuple(out))

    def mlem_packed(self, A: Matrix, y, s, x, niter: int, use_graph: bool = True, loglik: bool = False,
                    kernel_times: bool = False, stream=None):
        """MLEM iterations with A's delta-coded FP16 copy (A.to_packed()); as
        mlem_half()."""
        assert A.pword is not None, "call A.to_packed() first"
        ll = (C.c_double * max(niter, 1))() if loglik else None
        kt = (C.c_float * max(2 * niter, 1))() if kernel_times else None
        opts = raptr_mlem_opts(1 if use_graph else 0, C.cast(ll, C.POINTER(C.c_double)) if loglik else None,
                               C.cast(kt, C.POINTER(C.c_float)) if kernel_times else None, _ptr(A.row_rank))
        _check(lib().raptr_mlem_packed(self._h, A.m, A.n, _ptr(A.pseg), _ptr(A.panchor), _ptr(A.pword),
                                       _ptr(A.rscale), _ptr(A.tseg), _ptr(A.tanchor), _ptr(A.tword), _ptr(y),
                                       _ptr(s), _ptr(x), niter, C.byref(opts), _stream(stream)))
        out = []
        if loglik:
            out.append(np.array(ll[:niter]))
        if kernel_times:
            out.append(np.array(kt[:2 * niter], np.float64).reshape(niter, 2))
        return None if not out else (out[0] if len(out) == 1 else tuple(out))

    def _batch_arrays(self, A: Matrix, half: bool):
        if not A.has_transpose:
            A.transpose()
        if half:
            if A.hval is None:
                A.to_half()
            return 1, _ptr(A.hval), _ptr(A.rscale), _ptr(A.htval)
        return 0, _ptr(A.val), None, _ptr(A.tval)

    def mlem_batch(self, A: Matrix, Y, s, X, niter: int, frame_tile: int = 0, half: bool = True,
                   use_graph: bool = True, kernel_times: bool = False, stream=None):
        """MLEM for K frames together: Y (m, K) and X (n, K) float32,
        row-major (frame-minor); s the one normalised sensitivity.  Returns
        the (niter, 2) pass times with kernel_times, else None."""
        K = int(X.shape[1])
        assert Y.shape == (A.m, K) and X.shape == (A.n, K) and X.is_contiguous() and Y.is_contiguous()
        vt, val, rsc, tval = self._batch_arrays(A, half)
        kt = (C.c_float * max(2 * niter, 1))() if kernel_times else None
        opts = raptr_mlem_opts(1 if use_graph else 0, None, C.cast(kt, C.POINTER(C.c_float)) if kernel_times else None,
                               None)
        _check(lib().raptr_mlem_batch(self._h, A.m, A.n, K, vt, _ptr(A.row_ptr), _ptr(A.col), val, rsc,
                                      _ptr(A.col_ptr), _ptr(A.row_idx), tval, _ptr(A.row_rank), _ptr(Y), _ptr(s),
                                      _ptr(X), niter, frame_tile, C.byref(opts), _stream(stream)))
        return np.array(kt[:2 * niter], np.float64).reshape(niter, 2) if kernel_times else None

    def batch_autotune(self, A: Matrix, Y, s, X, half: bool = True, stream=None):
        """(best frame tile, {tile: ms per iteration}) for these frames."""
        K = int(X.shape[1])
        vt, val, rsc, tval = self._batch_arrays(A, half)
        best = C.c_int32(0)
        ms = (C.c_float * 5)()
        _check(lib().raptr_mlem_batch_autotune(self._h, A.m, A.n, K, vt, _ptr(A.row_ptr), _ptr(A.col), val, rsc,
                                               _ptr(A.col_ptr), _ptr(A.row_idx), tval, _ptr(A.row_rank), _ptr(Y),
                                               _ptr(s), _ptr(X), C.byref(best), ms, _stream(stream)))
        return best.value, {t: float(v) for t, v in zip((4, 8, 16, 32, 64), ms) if v >= 0}

    def mlem_f64(self, A: Matrix, y, s64, x64, niter: int, loglik: bool = False, stream=None):
        """MLEM iterations with FP64 vectors (x64, s64: float64 tensors; s64
        normalised to sum 1) over the FP32 matrix and its transpose."""
        if not A.has_transpose:
            A.transpose(stream)
        ll = (C.c_double * max(niter, 1))() if loglik else None
        _check(lib().raptr_mlem_f64(self._h, A.m, A.n, _ptr(A.row_ptr), _ptr(A.col), _ptr(A.val), _ptr(A.col_ptr),
                                    _ptr(A.row_idx), _ptr(A.tval), _ptr(A.row_rank), _ptr(y), _ptr(s64), _ptr(x64),
                                    niter, C.cast(ll, C.POINTER(C.c_double)) if loglik else None,
                                    _stream(stream)))
        return np.array(ll[:niter]) if loglik else None


class Server:
    """Serving loop (raptr_server): submit reconstructions of any geometry
    at any time; they run with continuous batching on one GPU, with system
    matrices cached in HBM."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 100 << 30, max_frames: int = 64,
                 keep_fp32: bool = False):
        o = raptr_server_opts(int(hbm_budget_bytes), int(max_frames), 1 if keep_fp32 else 0)
        h = VP()
        _check(lib().raptr_server_create(device, C.byref(o), C.byref(h)))
        self._h = h

    def submit(self, geom: Geometry, y, n_iter: int, nrays: int, seed: int) -> int:
        """Queues a reconstruction; y holds float32 counts of all channels."""
        y = np.ascontiguousarray(y, np.float32)
        if y.size != geom.n_channels:
            raise ValueError("y must hold one count per channel of the geometry")
        gs = geom_struct(geom)
        rid = C.c_int64(0)
        _check(lib().raptr_server_submit(self._h, C.byref(gs), nrays, seed, y.ctypes.data, n_iter, C.byref(rid)))
        return rid.value

    def wait(self, rid: int, n_voxels: int, timeout_ms: int = -1):
        """(image, stats) of a request; RaptrError on failure or timeout."""
        x = np.empty(n_voxels, np.float32)
        st = raptr_request_stats()
        _check(lib().raptr_server_wait(self._h, rid, x.ctypes.data, timeout_ms, C.byref(st)))
        return x, {k: getattr(st, k) for k, _ in raptr_request_stats._fields_}

    def stats(self) -> dict:
        st = raptr_server_stats()
        _check(lib().raptr_server_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in raptr_server_stats._fields_}

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            lib().raptr_server_destroy(h)
            self._h = None

    def __del__(self):
        self.close()


# -- context-free operations ---------------------------------------------------


def packed_words(seg, count: int) -> int:
    """Words of delta-coded runs whose quad offsets are seg (count + 1)."""
    return int(seg[count].item()) * 4


def pack_half(ptr, idx, hv, stream=None):
    """Delta-coded FP16 runs of (ptr, idx, hv) (raptr_pack_half): returns
    (seg, anchor, words) as device tensors (words as int32 bit patterns)."""
    torch = _torch()
    count = ptr.numel() - 1
    dev = ptr.device
    seg = torch.empty(count + 1, dtype=torch.int64, device=dev)
    anchor = torch.empty(max(count, 1), dtype=torch.int32, device=dev)
    nw = I64()
    _check(lib().raptr_pack_half(count, _ptr(ptr), _ptr(idx), _ptr(hv), _ptr(seg), _ptr(anchor), None, 0,
                                 C.byref(nw), _stream(stream)))
    words = torch.empty(max(nw.value, 4), dtype=torch.int32, device=dev)
    _check(lib().raptr_pack_half(count, _ptr(ptr), _ptr(idx), _ptr(hv), _ptr(seg), _ptr(anchor), _ptr(words),
                                 words.numel(), C.byref(nw), _stream(stream)))
    return seg, anchor[:count], words[:nw.value]


def sensitivity_half(A: Matrix, stream=None):
    """(FP64 column sums of A's FP16 copy, FP32 image normalised to sum 1)."""
    torch = _torch()
    s64 = torch.empty(A.n, dtype=torch.float64, device=A.row_ptr.device)
    s32 = torch.empty(A.n, dtype=torch.float32, device=A.row_ptr.device)
    _check(lib().raptr_sensitivity_half(A.n, _ptr(A.col_ptr), _ptr(A.row_idx), _ptr(A.htval), _ptr(A.pscale),
                                        _ptr(s64), _ptr(s32), _stream(stream)))
    return s64, s32

def spmv(op: int, m: int, n: int, row_ptr, col, val, x, alpha=1.0, beta=0.0, y=None, stream=None):
    """CSRmv: y = alpha*op(A)*x + beta*y."""
    torch = _torch()
    if y is None:
        y = torch.zeros(m if op == OP_N else n, dtype=torch.float32, device=x.device)
    _check(lib().raptr_spmv(op, m, n, _ptr(row_ptr), _ptr(col), _ptr(val), alpha, _ptr(x), beta, _ptr(y),
                            _stream(stream)))
    return y


def sensitivity(A: Matrix, stream=None, use_transpose: bool = True):
    """(FP64 column sums, FP32 image normalised to sum 1), through A's
    transpose when it has one (raptr_sensitivity_csc) unless use_transpose
    is False."""
    torch = _torch()
    s64 = torch.empty(A.n, dtype=torch.float64, device=A.row_ptr.device)
    s32 = torch.empty(A.n, dtype=torch.float32, device=A.row_ptr.device)
    if use_transpose and A.has_transpose and A.tval is not None:
        _check(lib().raptr_sensitivity_csc(A.n, _ptr(A.col_ptr), _ptr(A.tval), _ptr(s64), _ptr(s32),
                                           _stream(stream)))
    else:
        _check(lib().raptr_sensitivity(A.m, A.n, _ptr(A.row_ptr), _ptr(A.col), _ptr(A.val), _ptr(s64), _ptr(s32),
                                       _stream(stream)))
    return s64, s32


def mlem_project(A: Matrix, y, x, c, ll=None, stream=None):
    _check(lib().raptr_mlem_project(A.m, _ptr(A.row_ptr), _ptr(A.col), _ptr(A.val), _ptr(y), _ptr(x), _ptr(c),
                                    _ptr(ll), _stream(stream)))


def mlem_forward(A: Matrix, y, x, e, ll=None, stream=None):
    """e = y / (A x) (0 where y == 0), laid out as mlem_back(A, ...) reads it:
    in A's back-projection order when its transpose has one (e[row_rank[i]]
    for row i), else by row."""
    if A.row_rank is not None:
        _check(lib().raptr_mlem_forward_ordered(A.m, _ptr(A.row_ptr), _ptr(A.col), _ptr(A.val), _ptr(y), _ptr(x),
                                                _ptr(A.row_rank), _ptr(e), _ptr(ll), _stream(stream)))
        return
    _check(lib().raptr_mlem_forward(A.m, _ptr(A.row_ptr), _ptr(A.col), _ptr(A.val), _ptr(y), _ptr(x), _ptr(e),
                                    _ptr(ll), _stream(stream)))


def mlem_back(A: Matrix, e, c, stream=None):
    assert A.has_transpose, "call A.transpose() first"
    _check(lib().raptr_mlem_back(A.n, _ptr(A.col_ptr), _ptr(A.row_idx), _ptr(A.tval), _ptr(e), _ptr(c),
                                 _stream(stream)))


def csr_transpose(m: int, n: int, row_ptr, col, val, stream=None):
    torch = _torch()
    cp = torch.empty(n + 1, dtype=torch.int64, device=row_ptr.device)
    ri = torch.empty(max(col.numel(), 1), dtype=torch.int32, device=row_ptr.device)
    tv = torch.empty(max(col.numel(), 1), dtype=torch.float32, device=row_ptr.device)
    _check(lib().raptr_csr_transpose(m, n, _ptr(row_ptr), _ptr(col), _ptr(val), _ptr(cp), _ptr(ri), _ptr(tv),
                                     _stream(stream)))
    return cp, ri[:col.numel()], tv[:col.numel()]


def csr_transpose_ordered(m: int, n: int, row_ptr, col, val, order, stream=None):
    """CSC with the rows taken in `order` (a permutation of range(m)); the
    returned index array holds positions k in that order, ascending within
    each column."""
    torch = _torch()
    cp = torch.empty(n + 1, dtype=torch.int64, device=row_ptr.device)
    ri = torch.empty(max(col.numel(), 1), dtype=torch.int32, device=row_ptr.device)
    tv = torch.empty(max(col.numel(), 1), dtype=torch.float32, device=row_ptr.device)
    _check(lib().raptr_csr_transpose_ordered(m, n, _ptr(row_ptr), _ptr(col), _ptr(val), _ptr(order), _ptr(cp),
                                             _ptr(ri), _ptr(tv), _stream(stream)))
    return cp, ri[:col.numel()], tv[:col.numel()]


def mlem_update(x, c, s, acc, stream=None):
    _check(lib().raptr_mlem_update(x.numel(), _ptr(x), _ptr(c), _ptr(s), _ptr(acc), _stream(stream)))


def divides(res, a, b, stream=None):
    _check(lib().raptr_divides(_ptr(res), _ptr(a), _ptr(b), res.numel(), _stream(stream)))


def divides_multiplies(res, a, b, c, stream=None):
    _check(lib().raptr_divides_multiplies(_ptr(res), _ptr(a), _ptr(b), _ptr(c), res.numel(), _stream(stream)))


def scales(x, alpha: float, stream=None):
    _check(lib().raptr_scales(_ptr(x), alpha, x.numel(), _stream(stream)))


def vsum(x, stream=None) -> float:
    out = C.c_double()
    _check(lib().raptr_sum(_ptr(x), x.numel(), C.byref(out), _stream(stream)))
    return out.value


def coo2csr(rows, m: int, stream=None):
    torch = _torch()
    rp = torch.empty(m + 1, dtype=torch.int64, device=rows.device)
    _check(lib().raptr_coo2csr(_ptr(rows), rows.numel(), m, _ptr(rp), _stream(stream)))
    return rp


def csr2ecsr(yrow, csr, stream=None):
    torch = _torch()
    out = torch.empty(yrow.numel() + 1, dtype=torch.int64, device=csr.device)
    _check(lib().raptr_csr2ecsr(_ptr(out), _ptr(yrow), yrow.numel(), _ptr(csr), csr.numel() - 1, _stream(stream)))
    return out


def kernel_launches() -> int:
    """Kernels launched by the library in this process so far."""
    return lib().raptr_kernel_launches()


def trim_memory(device: int = -1) -> None:
    """Returns the device blocks the library keeps for reuse (freed
    matrices, transpose staging) to the driver; -1: every device."""
    _check(lib().raptr_trim_memory(device))


def reco_host(geom: Geometry, y: np.ndarray, nrays: int, seed: int, niter: int, sens: Optional[np.ndarray] = None,
              x0: Optional[np.ndarray] = None, device: int = 0):
    """The reco flow from host arrays: returns (x, stats dict)."""
    gs = geom_struct(geom)
    y = np.ascontiguousarray(y, np.float32)
    assert y.size == geom.n_channels
    x = np.zeros(geom.n_voxels, np.float32)
    st = raptr_reco_stats()
    sp = None if sens is None else np.ascontiguousarray(sens, np.float32)
    xp = None if x0 is None else np.ascontiguousarray(x0, np.float32)
    _check(lib().raptr_reco_host(C.byref(gs), device, y.ctypes.data, nrays, seed, niter,
                                 None if sp is None else sp.ctypes.data, None if xp is None else xp.ctypes.data,
                                 x.ctypes.data, C.byref(st)))
    stats = {f: getattr(st, f) for f, _ in raptr_reco_stats._fields_}
    return x, stats


__all__ = [
    "pack_half", "packed_words", "Geometry", "SMALL", "FULL", "FINE", "WORKLOADS", "epet_geometry", "phantom", "poisson_measurement", "Context",
    "Matrix", "spmv", "sensitivity", "mlem_project", "mlem_forward", "mlem_back", "csr_transpose", "mlem_update", "divides", "divides_multiplies", "scales",
    "vsum", "coo2csr", "csr2ecsr", "reco_host", "lib", "RaptrError", "OP_N", "OP_T", "trim_memory",
]
