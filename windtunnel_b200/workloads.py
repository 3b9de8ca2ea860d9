"""The benchmark channels: lattice, parameters and body of each workload.

* `channel256` — 256x128x128 D3Q19 channel, the seeded 20000-triangle
  superellipsoid hull (80x30x24 cells at scale 80, bumps of at most 2
  cells) voxelised at 160 cells along its length and placed at 15 degrees
  of yaw, u0 = 0.06, Re = 2000 on the length (tau = 0.5072), TRT
  Lambda = 3/16, Smagorinsky Cs = 0.1, free-slip side planes, seeded
  +-1e-4 velocity noise.
* `channel512` — the same body at scale 160 in a 512x192x192 channel.
* `sphere128` — 128x64x64 channel, sphere r = 8 at (32, 32, 32), Re = 100
  (a steady wake).

`hull_triangles` gives the oriented triangle soup (host arithmetic only),
`hull_grid` its Voxel.build on the GPU, `placement` the transform inputs of
the lookup (js/shapes.js:353-388, :473-486), and `channel_lattice` a
windtunnel_b200.LBM set up with all of it (voxelize through the device
lookup, seeded initial state).
"""
from __future__ import annotations

import math

WORKLOADS = {
    "channel256": dict(
        name="256x128x128 D3Q19 channel, yawed superellipsoid hull",
        nx=256, ny=128, nz=128, u0=0.06, tau=0.5072, csm=0.1, lam=3 / 16, les=True,
        side_bc="freeslip", body=dict(semi=(0.5, 0.1875, 0.15), exponent=2.5, res=160,
                                      scale=80.0, yaw_deg=15.0), seed=1234, amp=1e-4,
        accuracy_steps=10000, accuracy_window=2000),
    "sphere128": dict(
        name="128x64x64 D3Q19 channel, sphere r=8 at (32,32,32), Re=100 (steady wake)",
        nx=128, ny=64, nz=64, u0=0.05, tau=0.524, csm=0.1, lam=3 / 16, les=True,
        side_bc="freeslip", sphere=(32.0, 32.0, 32.0, 8.0), seed=1234, amp=1e-4,
        accuracy_steps=8000, accuracy_window=1000),
    "channel512": dict(
        name="512x192x192 D3Q19 channel, yawed superellipsoid hull x2",
        nx=512, ny=192, nz=192, u0=0.06, tau=0.5072, csm=0.1, lam=3 / 16, les=True,
        side_bc="freeslip", body=dict(semi=(0.5, 0.1875, 0.15), exponent=2.5, res=160,
                                      scale=160.0, yaw_deg=15.0), seed=1234, amp=1e-4,
        accuracy_steps=8000, accuracy_window=2000),
}

_TRIS: dict = {}
_GRIDS: dict = {}


def hull_triangles(body: dict, seed: int):
    """The seeded hull mesh, oriented and length-normalised (Shapes.orient)."""
    from .mesh import hull_mesh, orient
    key = (body["semi"], body["exponent"], seed)
    if key not in _TRIS:
        tris = hull_mesh(semi=body["semi"], exponent=body["exponent"], seed=seed)
        orient(tris, 0, 1)
        _TRIS[key] = tris
    return _TRIS[key]


def hull_grid(wl: dict):
    """Voxel.build of the workload's hull on the current CUDA device (cached)."""
    from .mesh import voxel_build
    b = wl["body"]
    key = (b["semi"], b["exponent"], b["res"], wl["seed"])
    if key not in _GRIDS:
        _GRIDS[key] = voxel_build(hull_triangles(b, wl["seed"]), b["res"])
    return _GRIDS[key]


def placement(wl: dict, ext) -> tuple[list, list, dict]:
    """(M, P, box): yaw rotation, position (0.36 nx, ny/2, nz/2) and the
    voxelize scan box of the workload's body with half extents `ext`."""
    from .bodies import body_box, body_matrix
    b = wl["body"]
    M = body_matrix(math.radians(b["yaw_deg"]), 0.0)
    P = [0.36 * wl["nx"], 0.5 * wl["ny"], 0.5 * wl["nz"]]
    return M, P, body_box(M, ext, b["scale"], P)


def set_params(sim, wl: dict) -> None:
    sim.set_params(u0=wl["u0"], tau=wl["tau"], csm=wl["csm"], les=int(wl["les"]),
                   **{"lambda": wl["lam"]})


def channel_lattice(wl: dict, storage: str = "f32", math_mode: str = "fast",
                    kernel: str = "auto"):
    """A windtunnel_b200.LBM holding the workload, ready to step."""
    from .lbm import LBM, sphere_box, sphere_inside
    sim = LBM(wl["nx"], wl["ny"], wl["nz"], storage=storage, math=math_mode,
              side_bc=wl["side_bc"], kernel=kernel)
    set_params(sim, wl)
    if "sphere" in wl:
        sim.voxelize(sphere_inside(*wl["sphere"]), sphere_box(*wl["sphere"]))
    else:
        vg = hull_grid(wl)
        M, P, box = placement(wl, vg.ext)
        sim.voxelize_grid(vg.grid, vg.min, vg.inv, M, P, wl["body"]["scale"], box)
    sim.init_eq_noise(wl["seed"], wl["amp"])
    return sim
