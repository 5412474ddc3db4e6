"""Generates tests/golden/*.npz from the reference's own code.

Run in a checkout where the reference sources are present (oracle/Makefile
builds oracle/_ref/libraptr_ref.so from them):

    python tests/golden/make_golden.py

Every array here is produced by reference code instantiated on the host
(getWorkqueue, intersectionLength, the Trafo functors, cooSort, the
mlemOperations, convertCsr2Ecsr); the ray unit-cube coordinates come from the
Philox4x32-10 stream (key = (seed, channel), counter = (ray, 0|1, 0, 0)).
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from raptr_b200 import config as cfg  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
SEED = 1251


def ref_rows(g, lst, nrays, seed):
    R = O.ref()
    U = np.stack([np.stack([O.ray_uniforms(seed, int(c), r) for r in range(nrays)]) for c in lst]).astype(np.float32)
    U = np.ascontiguousarray(U)
    cap = int(len(lst) * np.prod(g.grid_n))
    oc = np.zeros(cap, np.int32)
    ov = np.zeros(cap, np.int32)
    oval = np.zeros(cap, np.float32)
    n = R.ref_sysmat(C.byref(O.to_ogeom(g)), np.ascontiguousarray(lst, np.int32), len(lst), nrays, U, cap, oc, ov, oval)
    return oc[:n], ov[:n], oval[:n]


def ref_workqueue(g, lst, cursor, n):
    R = O.ref()
    cap = max(n, 1)
    oc = np.zeros(cap, np.int32)
    ov = np.zeros(cap, np.int32)
    li, vi = C.c_int32(cursor[0]), C.c_int32(cursor[1])
    k = R.ref_workqueue(C.byref(O.to_ogeom(g)), np.ascontiguousarray(lst, np.int32), len(lst), C.byref(li),
                        C.byref(vi), n, oc, ov)
    return oc[:k], ov[:k], (li.value, vi.value)


def main():
    O.build()
    assert O.ref_available(), "reference harness not built (reference sources missing?)"
    R = O.ref()
    out = {}

    # System-matrix rows (keep-zeros structure) of the small geometry.
    g = cfg.SMALL
    lst = np.array([0, 17, 5000, 71234, 142804], np.int32)
    c, v, val = ref_rows(g, lst, 100, SEED)
    out["small_list"], out["small_cnl"], out["small_vxl"], out["small_val"] = lst, c, v, val

    # Rows of the full geometry (fewer rays to keep the fixture small).
    g2 = cfg.FULL
    lst2 = np.array([12345, 2570490, 5140979], np.int32)
    c2, v2, val2 = ref_rows(g2, lst2, 64, SEED)
    out["full_list"], out["full_cnl"], out["full_vxl"], out["full_val"] = lst2, c2, v2, val2

    # Resumable workqueue: limited chunks from a cursor (prefix property of
    # src/tests/test_getWorkqueue.cu:206-218).
    wl = np.array([3, 99, 1000], np.int32)
    chunks = []
    cur = (0, 0)
    for n in (1000, 2500, 7, 50000):
        cc, vv, cur = ref_workqueue(g, wl, cur, n)
        chunks.append((cc, vv, cur))
    out["wq_list"] = wl
    out["wq_sizes"] = np.array([1000, 2500, 7, 50000], np.int64)
    out["wq_cnl"] = np.concatenate([x[0] for x in chunks])
    out["wq_vxl"] = np.concatenate([x[1] for x in chunks])
    out["wq_counts"] = np.array([x[0].size for x in chunks], np.int64)
    out["wq_cursors"] = np.array([x[2] for x in chunks], np.int64)

    # Crystal transforms (in-place) of random unit-cube points, both heads.
    rng = np.random.Generator(np.random.PCG64(7))
    pts = rng.random((16, 3)).astype(np.float32)
    ids = rng.integers(0, [g2.na, 13, 13], size=(16, 3)).astype(np.int32)
    tr = np.zeros((2, 16, 3), np.float32)
    for det in (0, 1):
        for i in range(16):
            o = np.zeros(3, np.float32)
            R.ref_trafo(C.byref(O.to_ogeom(g2)), det, 1, int(ids[i, 0]), int(ids[i, 1]), int(ids[i, 2]),
                        np.ascontiguousarray(pts[i]), o)
            tr[det, i] = o
    out["trafo_pts"], out["trafo_ids"], out["trafo_out"] = pts, ids, tr

    # intersectionLength on rays of the full geometry against nearby voxels.
    rays = O.rays(g2, np.array([2570490], np.int32), 8, SEED)[0]
    boxes, lens = [], []
    for r in rays:
        vox, _ = O.walk_ray(g2, r)
        for vv_ in vox[::7]:
            ix, iy, iz = O.voxel_split(g2, int(vv_))
            b = np.array([g2.grid_o[0] + ix * np.float32(g2.grid_d[0]), 0, 0, 0, 0, 0], np.float32)
            box = np.zeros(6, np.float32)
            for d, i in enumerate((ix, iy, iz)):
                box[d] = np.float32(np.float32(g2.grid_o[d]) + np.float32(i) * np.float32(g2.grid_d[d]))
                box[3 + d] = np.float32(np.float32(g2.grid_o[d]) + np.float32(i + 1) * np.float32(g2.grid_d[d]))
            del b
            boxes.append(box)
            lens.append(R.ref_intersection_length(box, np.ascontiguousarray(r)))
    out["il_rays"] = np.repeat(rays, [len(O.walk_ray(g2, r)[0][::7]) for r in rays], axis=0)
    out["il_boxes"] = np.array(boxes, np.float32)
    out["il_len"] = np.array(lens, np.float32)

    # MLEM operations known answer (src/tests/test_mlemOperations.cu:59-109):
    # A=(i+1)^2, B=10, C=i+1.
    n = 10
    A = ((np.arange(n) + 1) ** 2).astype(np.float32)
    B = np.full(n, 10, np.float32)
    Cc = (np.arange(n) + 1).astype(np.float32)
    D = np.zeros(n, np.float32)
    R.ref_divides(D, A.copy(), Cc.copy(), n)
    out["mlem_divides"] = D.copy()
    R.ref_divides_multiplies(D, A.copy(), B.copy(), Cc.copy(), n)
    out["mlem_divmul"] = D.copy()
    out["mlem_sum"] = np.array([R.ref_sum(D.copy(), n)], np.float32)
    S = D.copy()
    R.ref_scales(S, np.float32(1.0 / out["mlem_sum"][0]), n)
    out["mlem_scaled"] = S

    np.savez_compressed(os.path.join(OUT, "reference_golden.npz"), **out)
    print("wrote", os.path.join(OUT, "reference_golden.npz"), {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
