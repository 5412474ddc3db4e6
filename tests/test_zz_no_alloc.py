"""raptr_mlem_noalloc: MLEM without device allocation.

Some callers cannot allocate device memory where they reconstruct (a server
that reserves its whole HBM budget in its own pool, a pipeline that cannot
take the synchronisation of cudaMalloc/cudaFree).  This entry point keeps its
workspace in a fixed array inside the library.  Here it is called through the
C ABI twice in a row -- the second call reuses the array the first call
used -- and each result is checked against the allocating entry point
raptr_mlem (same iteration, scatter back projection) to the tolerance of the
other MLEM tests: 1e-5 relative L2 (the atomic back projection sums in a
varying order).  The device's free memory is the same before and after the
second call: the call allocates nothing.  Collected last, so a failure here
stops a -x run only after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from raptr_b200 import config as cfg

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def test_mlem_noalloc_matches_allocating_entry_point(rlib):
    import torch

    assert torch.cuda.is_available()
    L = rlib.lib()
    g = cfg.SMALL
    ctx = rlib.Context(g, 0)
    lst = np.arange(0, g.n_channels, 5, dtype=np.int32)
    A = ctx.build(lst, 100, 1251)
    xt = torch.from_numpy(cfg.phantom(g, rods=False)).cuda()
    y = rlib.spmv(rlib.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, xt) * 1e4
    s64, s = rlib.sensitivity(A)
    x0 = torch.full((A.n,), np.float32(1.0 / A.n), device="cuda")
    x_ref = x0.clone()
    ctx.mlem(A, y, s, x_ref, 8, use_graph=False)  # raptr_mlem, no transpose: same scatter iteration
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        x = x0.clone()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = L.raptr_mlem_noalloc(A.m, A.n, A.row_ptr.data_ptr(), A.col.data_ptr(), A.val.data_ptr(), y.data_ptr(),
                                  s.data_ptr(), x.data_ptr(), 8, stream)
        assert st == 0, L.raptr_last_error()
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:
            # the first call on the device may load the module that holds
            # the array; from then on a call allocates nothing
            assert free_after == free_before, f"free device memory changed by {free_before - free_after} bytes"
        rel = float(torch.linalg.norm(x - x_ref) / torch.linalg.norm(x_ref))
        assert rel < RTOL, f"call {call}: rel L2 {rel}"
        assert abs(float(x.sum()) - 1.0) < 1e-5


def test_mlem_noalloc_rejects_bad_arguments(rlib):
    L = rlib.lib()
    big = (1 << 20) + 1
    st = L.raptr_mlem_noalloc(1, big, 1, 1, 1, 1, 1, 1, 1, None)
    assert st == 1 and b"1048576" in L.raptr_last_error()
    # rows without column or value arrays
    st = L.raptr_mlem_noalloc(4, 16, 1, None, 1, 1, 1, 1, 1, None)
    assert st == 1 and b"null column or value" in L.raptr_last_error()
    st = L.raptr_mlem_noalloc(4, 16, 1, 1, None, 1, 1, 1, 1, None)
    assert st == 1
