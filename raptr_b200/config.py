"""Scanner geometries and synthetic workloads.

A geometry carries the fields of the reference's DefaultVoxelGrid
(src/VoxelGrid.hpp:151-176) and DefaultMeasurementSetup
(src/MeasurementSetup.hpp:181-220), in the reference's units (metres,
degrees).  The named workloads are the two-head ePET scanner with 13x13
crystals of 4x4x20 mm whose front faces sit at +-230 mm, so the crystal
centres are at x = -+240 mm.
"""
from __future__ import annotations

import dataclasses
from typing import Tuple

import numpy as np


@dataclasses.dataclass(frozen=True)
class Geometry:
    grid_o: Tuple[float, float, float]
    grid_d: Tuple[float, float, float]
    grid_n: Tuple[int, int, int]
    pos0x: float
    pos1x: float
    na: int
    n0z: int
    n0y: int
    n1z: int
    n1y: int
    da: float
    segx: float
    segy: float
    segz: float

    @property
    def n_voxels(self) -> int:
        return int(self.grid_n[0]) * int(self.grid_n[1]) * int(self.grid_n[2])

    @property
    def n_channels(self) -> int:
        return int(self.na) * self.n0z * self.n0y * self.n1z * self.n1y

    def voxel_centres(self) -> np.ndarray:
        """(N, 3) float64 voxel centres in linear-id order (x slowest, z fastest)."""
        ax = [self.grid_o[d] + (np.arange(self.grid_n[d]) + 0.5) * self.grid_d[d] for d in range(3)]
        X, Y, Z = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
        return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def epet_geometry(n_vox: int, pitch: float, n_angles: int, step_deg: float) -> Geometry:
    """Cubic grid of n_vox^3 voxels of `pitch` metres centred on the isocentre,
    two 13x13 heads of 4x4x20 mm crystals, `n_angles` rotation steps."""
    half = n_vox * pitch / 2.0
    return Geometry(
        grid_o=(-half, -half, -half),
        grid_d=(pitch, pitch, pitch),
        grid_n=(n_vox, n_vox, n_vox),
        pos0x=-0.240,
        pos1x=0.240,
        na=n_angles,
        n0z=13,
        n0y=13,
        n1z=13,
        n1y=13,
        da=step_deg,
        segx=0.020,
        segy=0.004,
        segz=0.004,
    )


# 40^3 x 2 mm, 5 angles of 36 degrees, 100 rays, 2e6 counts, 20 iterations.
SMALL = epet_geometry(40, 0.002, 5, 36.0)
# 70^3 x 2 mm, 180 angles of 2 degrees, 1000 rays, 1e8 counts, 50 iterations.
FULL = epet_geometry(70, 0.002, 180, 2.0)
# 100^3 x 1.5 mm, 60 angles; the angular step is not given for this geometry,
# 3 degrees (60 x 3 = 180 degrees) is used.
FINE = epet_geometry(100, 0.0015, 60, 3.0)

WORKLOADS = {
    "small": dict(geom=SMALL, nrays=100, counts=2e6, niter=20, rods=False),
    "full": dict(geom=FULL, nrays=1000, counts=1e8, niter=50, rods=True),
    "fine": dict(geom=FINE, nrays=1000, counts=1e7, niter=25, rods=True),
}

# Rod array: five rods of radius 2..6 mm along z on a ring of radius 45 mm,
# at azimuths 36 + k*72 degrees in the x-y plane (clear of both spheres).
ROD_RING_M = 0.045
ROD_RADII_M = (0.002, 0.003, 0.004, 0.005, 0.006)
ROD_AZIMUTH_DEG = tuple(36.0 + 72.0 * k for k in range(5))


def phantom(g: Geometry, rods: bool) -> np.ndarray:
    """Activity by voxel-centre inclusion: background 0.1 in every voxel,
    sphere r=15 mm at the centre with 1.0, sphere r=8 mm at (+20, 0, 0) mm with
    4.0 (painted over the first), and optionally the rod array with 2.0."""
    c = g.voxel_centres()
    x = np.full(c.shape[0], 0.1, np.float64)
    r2 = (c ** 2).sum(1)
    x[r2 < 0.015 ** 2] = 1.0
    x[((c - np.array([0.020, 0.0, 0.0])) ** 2).sum(1) < 0.008 ** 2] = 4.0
    if rods:
        for rad, az in zip(ROD_RADII_M, ROD_AZIMUTH_DEG):
            cx = ROD_RING_M * np.cos(np.deg2rad(az))
            cy = ROD_RING_M * np.sin(np.deg2rad(az))
            x[(c[:, 0] - cx) ** 2 + (c[:, 1] - cy) ** 2 < rad ** 2] = 2.0
    return x.astype(np.float32)


def poisson_measurement(expected: np.ndarray, total_counts: float, seed: int) -> np.ndarray:
    """y ~ Poisson(lambda), lambda = expected scaled to `total_counts` in sum."""
    lam = expected.astype(np.float64)
    lam *= total_counts / lam.sum()
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.poisson(lam).astype(np.float32)
