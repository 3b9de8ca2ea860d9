"""Body placement on the host: the transform inputs of the occupancy lookup.

Mirrors the parts of js/shapes.js the solver consumes: Body._updateMat
(js/shapes.js:353-362, R = Ry(yaw) * Rz(pitch), row-major), Body.box
(js/shapes.js:473-486, the AABB the voxelize scan covers) and the
voxel-grid record of js/voxel.js:89-101. The lookup itself runs on the
device (wt_voxelize_grid).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class VoxelGrid:
    """Body-space occupancy grid, the record js/voxel.js:89-101 returns."""
    grid: np.ndarray          # uint8, shape (nz, ny, nx), index a + nx*(b + ny*c)
    cell: float
    min: list                 # [x, y, z] of the grid's min corner
    ext: list                 # half extents of the body in body space
    stats: dict = field(default_factory=dict)

    @property
    def inv(self) -> float:
        return 1 / self.cell

    @property
    def dims(self) -> tuple[int, int, int]:
        nz, ny, nx = self.grid.shape
        return nx, ny, nz


def body_matrix(yaw: float, pitch: float) -> list[float]:
    """Body -> world rotation, js/shapes.js:353-362 (yaw about y, then pitch about z)."""
    cy, sy = math.cos(yaw), math.sin(yaw)
    cp, sp = math.cos(pitch), math.sin(pitch)
    return [cy * cp, -cy * sp, sy,
            sp, cp, 0.0,
            -sy * cp, sy * sp, cy]


def body_box(M, ext, scale: float, pos) -> dict:
    """Tight lattice-space AABB plus 2 cells, js/shapes.js:473-486."""
    w = [scale * (abs(M[i * 3]) * ext[0] + abs(M[i * 3 + 1]) * ext[1] +
                  abs(M[i * 3 + 2]) * ext[2]) + 2 for i in range(3)]
    return {"x0": pos[0] - w[0], "x1": pos[0] + w[0],
            "y0": pos[1] - w[1], "y1": pos[1] + w[1],
            "z0": pos[2] - w[2], "z1": pos[2] + w[2]}


def superellipsoid_grid(semi=(0.5, 0.1875, 0.15), exponent: float = 2.5,
                        res: int = 160, pad: int = 2) -> VoxelGrid:
    """Occupancy of |x/a|^e + |y/b|^e + |z/c|^e <= 1 sampled at voxel centres.

    The grid follows js/voxel.js:53-68's framing: `res` cells along the
    longest axis, `pad` cells of margin, body centred in the padded grid.
    """
    a, b, c = semi
    span = 2 * max(semi)
    cell = span / res
    sx, sy, sz = 2 * a, 2 * b, 2 * c
    nx = max(3, math.ceil(sx / cell) + 2 * pad)
    ny = max(3, math.ceil(sy / cell) + 2 * pad)
    nz = max(3, math.ceil(sz / cell) + 2 * pad)
    mn = [-a - (nx * cell - sx) * 0.5, -b - (ny * cell - sy) * 0.5, -c - (nz * cell - sz) * 0.5]
    xs = mn[0] + (np.arange(nx) + 0.5) * cell
    ys = mn[1] + (np.arange(ny) + 0.5) * cell
    zs = mn[2] + (np.arange(nz) + 0.5) * cell
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    v = np.abs(X / a) ** exponent + np.abs(Y / b) ** exponent + np.abs(Z / c) ** exponent
    grid = (v <= 1.0).astype(np.uint8)
    return VoxelGrid(grid=grid, cell=cell, min=mn, ext=[a, b, c],
                     stats={"solid": int(grid.sum())})
