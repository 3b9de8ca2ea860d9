"""Matched set-ups of the CUDA path (windtunnel_b200.LBM) and the CPU oracle.

A case is a lattice, parameters, an occupancy and a seeded initial state,
applied identically to both sides so that their outputs can be compared.
"""
from __future__ import annotations

import numpy as np

from windtunnel_b200.lbm import sphere_box, sphere_inside

CFG0 = dict(nx=128, ny=64, nz=64, u0=0.05, tau=0.512, csm=0.1, lam=3 / 16,
            sphere=(32.0, 32.0, 32.0, 8.0), seed=1234, amp=1e-4)


def apply_case(sim, *, u0=0.05, tau=0.512, csm=0.1, lam=3 / 16, les=True, trt=True,
               side_bc="eq", sphere=None, ground=False, roadVel=0.0, wallVel=None,
               seed=1234, amp=1e-4, math=None):
    """Configure `sim` (LBM or OracleLBM) the same way on either side."""
    kw = dict(u0=u0, tau=tau, csm=csm, les=int(les), trt=int(trt), side_bc=side_bc)
    kw["lambda"] = lam
    if math is not None:
        kw["math"] = math
    sim.set_params(**kw)
    if sphere is not None:
        cx, cy, cz, r = sphere
        sim.voxelize(sphere_inside(cx, cy, cz, r), sphere_box(cx, cy, cz, r), ground,
                     wallVel, roadVel)
    elif ground or roadVel:
        sim.voxelize(lambda x, y, z: np.zeros_like(x, dtype=bool),
                     {"x0": 0, "y0": 0, "z0": 0, "x1": -1, "y1": -1, "z1": -1}, ground, None,
                     roadVel)
    if amp:
        sim.init_eq_noise(seed, amp)
    return sim


def spinning_sphere_wallvel(cx, cy, cz, omega):
    """wallVel closure of a sphere spinning about z (reference signature fn(x,y,z,out))."""
    def wall(x, y, z, out):
        rx, ry = x - cx, y - cy
        out[0] = -omega * ry
        out[1] = omega * rx
        out[2] = 0.0
        return True
    return wall


def rel_linf(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / scale)


def pair_average(series: np.ndarray) -> np.ndarray:
    """Average of consecutive steps, js/main.js:113-127 (cancels the odd/even oscillation)."""
    s = np.asarray(series, np.float64)
    return 0.5 * (s[1:] + s[:-1])


def oracle_channel(wl):
    """A benchmark channel (windtunnel_b200.workloads) on the CPU oracle: the
    hull voxelised by the oracle's Voxel.build (bit-identical to the GPU's),
    placed by the oracle's lookup, with the workload's parameters and seeded
    state."""
    from oracle.oracle import OracleLBM, lookup_mask, voxel_build
    from windtunnel_b200.workloads import hull_triangles, placement, set_params
    o = OracleLBM(wl["nx"], wl["ny"], wl["nz"], "f32", side_bc=wl["side_bc"])
    set_params(o, wl)
    b = wl["body"]
    grid, info = voxel_build(hull_triangles(b, wl["seed"]), b["res"])
    M, P, box = placement(wl, info["ext"])
    mask = lookup_mask(grid, info["min"], info["inv"], M, P, b["scale"], wl["nx"], wl["ny"],
                       wl["nz"], box)
    o.voxelize_mask(box, mask)
    o.init_eq_noise(wl["seed"], wl["amp"])
    return o
