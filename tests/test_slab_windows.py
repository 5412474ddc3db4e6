"""Dense slab windows of the system-matrix build, checked on the host.

The row kernel adds a row's ray lengths to dense slots without keys when
both crystals of the channel lie on opposite sides of the grid along x or z:
for each slab of that axis it bounds the voxels the rays can reach from the
crystal boxes' corners (csrc/kernels_sm.cu: crystal_boxes, slab_window, the
axis choice in sm_rows_kernel), widened by one voxel on each side.  Here
that computation is restated in float32 and checked against the voxels the
exact walk visits on the channel's rays (the oracle's walk over the same
Philox rays as the GPU's): every visited voxel lies inside its slab's
window with the one-voxel margin to spare (where the window is not clamped
at the grid's edge), and on the 40^3 and 70^3 workloads every sampled row
fits the dense slot limit."""
import numpy as np
import pytest

from raptr_b200 import config as cfg

F = np.float32
MAX_SLABS = 256


def dense_slots(h):
    return 3 * h if h <= 4096 else 2 * h


def boxes(O, g, cnl):
    ida, id0z, id0y, id1z, id1y = (int(v) for v in O.channel_split(g, cnl))
    corners = np.array([[c & 1, (c >> 1) & 1, (c >> 2) & 1] for c in range(8)], np.float32)
    out = []
    for det, (idz, idy) in enumerate(((id0z, id0y), (id1z, id1y))):
        p = O.trafo_f(g, det, ida, idz, idy, corners)
        centre = O.trafo_f(g, det, ida, idz, idy, np.full((1, 3), 0.5, np.float32))[0]
        out.append((p.min(0), p.max(0), centre))
    return out


def windows(g, b0, b1):
    """(axis, [(lo_u, hi_u, lo_v, hi_v) per slab]) as the row kernel computes
    them, or None where the row takes the hash table."""
    o = np.array(g.grid_o, F)
    d = np.array(g.grid_d, F)
    n = np.array(g.grid_n)
    lo = (b0[0], b1[0])
    hi = (b0[1], b1[1])
    ab = b1[2] - b0[2]
    first = 0 if abs(ab[0]) >= abs(ab[2]) else 2
    axis, sdir = None, 0
    for a in (first, 2 - first):
        if n[a] > MAX_SLABS:
            continue
        c0 = o[a]
        c1 = F(o[a] + F(F(n[a]) * d[a]))
        m = F(F(1e-6) * F(F(1.0) + F(abs(c0)) + F(abs(c1))))
        if F(hi[0][a] + m) < c0 and F(lo[1][a] - m) > c1:
            axis, sdir = a, 1
        elif F(hi[1][a] + m) < c0 and F(lo[0][a] - m) > c1:
            axis, sdir = a, -1
        if axis is not None:
            break
    if axis is None:
        return None
    p = 0 if sdir > 0 else 1
    plo, phi, qlo, qhi = lo[p], hi[p], lo[1 - p], hi[1 - p]
    u, v = (1, 2) if axis == 0 else (0, 1)
    out = []
    for s in range(n[axis]):
        cs = (F(o[axis] + F(F(s) * d[axis])), F(o[axis] + F(F(s + 1) * d[axis])))
        row = []
        for w in (u, v):
            wlo, whi = F(np.inf), F(-np.inf)
            for c in cs:
                t1 = F(F(c - phi[axis]) / F(qhi[axis] - phi[axis]))
                t2 = F(F(c - plo[axis]) / F(qlo[axis] - plo[axis]))
                for t in (t1, t2):
                    wlo = min(wlo, F(plo[w] + F(t * F(qlo[w] - plo[w]))))
                    whi = max(whi, F(phi[w] + F(t * F(qhi[w] - phi[w]))))
            a_ = int(np.floor(F(F(wlo - o[w]) / d[w]))) - 1
            b_ = int(np.floor(F(F(whi - o[w]) / d[w]))) + 1
            a_ = min(max(a_, 0), n[w] - 1)
            b_ = min(max(b_, 0), n[w] - 1)
            row += [a_, max(a_, b_)]
        out.append(tuple(row))
    return axis, out


# an off-centre grid whose origin, pitch and size differ per axis, 12 angles of 15 degrees
ANISO = cfg.Geometry(grid_o=(-0.061, -0.047, -0.039), grid_d=(0.002, 0.0025, 0.0018), grid_n=(60, 40, 48),
                     pos0x=-0.240, pos1x=0.240, na=12, n0z=13, n0y=13, n1z=13, n1y=13, da=15.0, segx=0.020,
                     segy=0.004, segz=0.004)


@pytest.mark.parametrize("which,level_h", [("small", 2048), ("full", 4096), ("fine", 8192), ("aniso", 4096)])
def test_walked_voxels_lie_inside_the_slab_windows(oracle, which, level_h):
    g = {"small": cfg.SMALL, "full": cfg.FULL, "fine": cfg.FINE, "aniso": ANISO}[which]
    O = oracle
    rng = np.random.default_rng(21)
    lst = rng.integers(0, g.n_channels, 24).astype(np.int32)
    rays = O.rays(g, lst, 40, 1251)
    n = np.array(g.grid_n)
    dense_rows = 0
    for k, cnl in enumerate(lst):
        b0, b1 = boxes(O, g, int(cnl))
        win = windows(g, b0, b1)
        assert win is not None  # the crystals of these workloads are always separated along x or z
        axis, rows = win
        u, v = (1, 2) if axis == 0 else (0, 1)
        wu = max(r[1] - r[0] + 1 for r in rows)
        wv = max(r[3] - r[2] + 1 for r in rows)
        dense_rows += int(n[axis] * wu * wv < dense_slots(level_h))
        for ray in rays[k]:
            vox, length = O.walk_ray(g, ray)
            for vid, L in zip(vox, length):
                if not L > 0:
                    continue
                ijk = (vid // (n[1] * n[2]), (vid // n[2]) % n[1], vid % n[2])
                lu, hu, lv, hv = rows[ijk[axis]]
                iu, iv = ijk[u], ijk[v]
                # inside, and one voxel inside where the window is not clamped at the grid edge
                assert (lu + 1 if lu > 0 else 0) <= iu <= (hu - 1 if hu < n[u] - 1 else n[u] - 1), (cnl, ijk)
                assert (lv + 1 if lv > 0 else 0) <= iv <= (hv - 1 if hv < n[v] - 1 else n[v] - 1), (cnl, ijk)
    if which in ("small", "full"):
        assert dense_rows == lst.size
