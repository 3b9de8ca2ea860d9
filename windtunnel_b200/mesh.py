"""Triangle-soup bodies: the seeded hull of the benchmark channels, the
reference's body-space orientation, and Voxel.build on the GPU.

* `hull_mesh` builds a closed superellipsoid hull with a seeded radial bump
  field as a float32 triangle soup (nine numbers per triangle), tessellated
  on a (u, v) grid.
* `orient` restates Shapes.orient (js/shapes.js:212-248): rotate to nose -x,
  up +y, centre, and scale the length to 1, writing through float32 as the
  reference's Float32Array does.
* `voxel_build` runs Voxel.build (js/voxel.js:48-232) on the current CUDA
  device through the C ABI (wt_voxel_build) and returns the grid with the
  fields of the reference's voxel object.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as W
from ._lib import lib


def _sgnpow(c: np.ndarray, m: float) -> np.ndarray:
    return np.sign(c) * np.abs(c) ** m


def hull_mesh(semi=(0.5, 0.1875, 0.15), exponent: float = 2.5, nu: int = 100, nv: int = 100,
              bumps: int = 16, bump_amp: float = 0.025, seed: int = 1234) -> np.ndarray:
    """Closed superellipsoid hull (semi-axes in body units, nose along -x) with
    `bumps` seeded Gaussian bumps of amplitude at most `bump_amp` displacing
    the surface radially; 2*nu*nv triangles as a float32 array of 9 per triangle."""
    rng = np.random.default_rng(seed)
    centres = rng.normal(size=(bumps, 3))
    centres /= np.linalg.norm(centres, axis=1, keepdims=True)
    amps = rng.uniform(-bump_amp, bump_amp, bumps)
    widths = rng.uniform(0.15, 0.4, bumps)
    m = 2.0 / exponent
    u = np.linspace(-np.pi, np.pi, nu + 1)[:-1]            # periodic
    v = np.linspace(-np.pi / 2, np.pi / 2, nv + 1)         # pole to pole
    V, U = np.meshgrid(v, u, indexing="ij")                # (nv+1, nu)
    cu, su = _sgnpow(np.cos(U), m), _sgnpow(np.sin(U), m)
    cv, sv = _sgnpow(np.cos(V), m), _sgnpow(np.sin(V), m)
    X = np.stack([semi[0] * cv * cu, semi[1] * cv * su, semi[2] * sv], axis=-1)
    # radial bump field, evaluated on the direction of each point
    d = X / np.maximum(np.linalg.norm(X, axis=-1, keepdims=True), 1e-12)
    disp = np.zeros(X.shape[:2])
    for c, a, w in zip(centres, amps, widths):
        disp += a * np.exp(-np.sum((d - c) ** 2, axis=-1) / (2 * w * w))
    X = X + d * disp[..., None]
    tris = []
    for j in range(nv):
        for i in range(nu):
            i2 = (i + 1) % nu
            p00, p01 = X[j, i], X[j, i2]
            p10, p11 = X[j + 1, i], X[j + 1, i2]
            tris.append((p00, p10, p11))
            tris.append((p00, p11, p01))
    return np.asarray(tris, np.float64).astype(np.float32).ravel()


def orient(P: np.ndarray, forward: int = 0, up: int = 1, flip: bool = False,
           ground: bool = False) -> float:
    """Shapes.orient (js/shapes.js:212-248) in place on a float32 soup; returns
    the length scale k. Rotation rows are (-f, u, -f x u); the length along x
    becomes 1 and the bounds are centred (or rest on y = 0 with ground)."""
    if forward == up:
        forward = (up + 1) % 3
    f = [0.0, 0.0, 0.0]
    u = [0.0, 0.0, 0.0]
    f[forward] = -1.0 if flip else 1.0
    u[up] = 1.0
    s = [f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0]]
    R = np.array([[-f[0], -f[1], -f[2]], u, [-s[0], -s[1], -s[2]]], np.float64)
    V = P.reshape(-1, 3).astype(np.float64)
    rot = V @ R.T
    lo, hi = rot.min(axis=0), rot.max(axis=0)
    P.reshape(-1, 3)[:] = rot.astype(np.float32)
    k = 1.0 / max(1e-9, hi[0] - lo[0])
    cx, cz = (lo[0] + hi[0]) * 0.5, (lo[2] + hi[2]) * 0.5
    cy = lo[1] if ground else (lo[1] + hi[1]) * 0.5
    V = P.reshape(-1, 3).astype(np.float64)
    V = (V - np.array([cx, cy, cz])) * k
    P.reshape(-1, 3)[:] = V.astype(np.float32)
    return k


@dataclass
class VoxelGrid:
    """The fields of Voxel.build's result (js/voxel.js:89-101)."""
    grid: np.ndarray          # [nz][ny][nx] uint8
    nx: int
    ny: int
    nz: int
    cell: float
    min: list
    inv: float
    ext: list
    centre: list
    bbox: list
    tris: int
    solid: int
    openness: float


def voxel_build(P: np.ndarray, res: int = 96) -> VoxelGrid:
    """Voxel.build(P, res) on the GPU (bit-identical to the reference)."""
    p = np.ascontiguousarray(P, np.float32).ravel()
    ntri = p.size // 9
    info = W.wt_voxel_info()
    L = lib()
    tp = p.ctypes.data_as(C.POINTER(C.c_float))
    rc = L.wt_voxel_dims(tp, ntri, int(res), C.byref(info))
    if rc < 0:
        raise W.WTError(rc, L.wt_voxel_last_error().decode())
    grid = np.zeros((info.nz, info.ny, info.nx), np.uint8)
    rc = L.wt_voxel_build(tp, ntri, int(res), grid.ctypes.data_as(C.POINTER(C.c_uint8)),
                          grid.size, C.byref(info))
    if rc < 0:
        raise W.WTError(rc, L.wt_voxel_last_error().decode())
    return VoxelGrid(grid=grid, nx=info.nx, ny=info.ny, nz=info.nz, cell=info.cell,
                     min=list(info.min), inv=info.inv, ext=list(info.ext),
                     centre=list(info.centre), bbox=list(info.bbox), tris=info.tris,
                     solid=info.solid, openness=info.openness)
