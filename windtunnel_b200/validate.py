"""The reference's validation page on the GPU path (test.html:35-95).

    python -m windtunnel_b200.validate [--math exact|fast] [--storage f32|f16dev|f64]

Runs the eleven bluff-body cases of test.html on a 96x44x44 lattice at the
page's Reynolds setting (tau = 0.5 + 10^(-1.1 - 2.3*0.62)): each body is
fitted, placed at (0.36 nx, ground ? 1 : ny/2, nz/2) with pitch -aoa,
voxelised through the analytic closure, stepped 400 times, and its Cd / Cl
are the plain means of the force over the next 300 steps over
(1/2 u0^2 A), A the frontal or (wings, airliner) planform area. The
reference's published values for the same runs (its README validation
table) are printed beside them.
"""
from __future__ import annotations

import argparse
import json
import math

from .lbm import LBM
from .shapes import Body
from .stats import block_stats

NX, NY, NZ, WARM, AVG = 96, 44, 44, 400, 300
TAU = 0.5 + math.pow(10, -1.1 - 2.3 * 0.62)

# (name, body, ground, aoa in degrees) -- test.html:36-48
CASES = [
    ("sphere", "sphere", False, 0), ("cube", "cube", False, 0),
    ("cylinder", "cylinder", False, 0), ("teardrop", "teardrop", False, 0),
    ("sedan", "sedan", True, 0), ("truck", "truck", True, 0),
    ("wing a=-8", "wing", False, -8), ("wing a=0", "wing", False, 0),
    ("wing a=8", "wing", False, 8), ("wing a=16", "wing", False, 16),
    ("airplane", "airplane", False, 2),
]

# The reference's measured values of these runs (its README validation table).
PUBLISHED = {"cylinder": {"cd": 1.13}, "cube": {"cd": 1.18}, "sphere": {"cd": 0.86},
             "sedan": {"cd": 1.12}, "truck": {"cd": 1.39}, "teardrop": {"cd": 1.02},
             "wing a=-8": {"cl": -0.26}, "wing a=0": {"cl": 0.01}, "wing a=8": {"cl": 0.42}}


def run_case(name: str, key: str, ground: bool, aoa: float, storage: str = "f32",
             math_mode: str = "exact") -> dict:
    sim = LBM(NX, NY, NZ, storage=storage, math=math_mode)
    sim.set_params(tau=TAU)
    b = Body(key)
    b.fit(NX, NY, NZ)
    b.pos = [NX * 0.36, 1 if ground else NY * 0.5, NZ * 0.5]
    b.pitch = -aoa * math.pi / 180
    sim.voxelize(b.make_test(), b.box(), ground)
    area = sim.planformArea if b.ref == "planform" else sim.frontalArea
    sim.step_forces(WARM)
    F = sim.step_forces(AVG)
    q = 0.5 * sim.u0 * sim.u0 * area
    sem = block_stats(F[:, 0] / q).sem   # blocking standard error of the mean drag
    out = {"case": name, "cd": float(F[:, 0].mean() / q), "cl": float(F[:, 1].mean() / q),
           "cd_sem": float(sem), "solid_cells": sim.solidCells, "area": area,
           "area_kind": "planform" if b.ref == "planform" else "frontal"}
    out["published"] = PUBLISHED.get(name, {})
    sim.close()
    return out


def run_all(storage: str = "f32", math_mode: str = "exact") -> list[dict]:
    return [run_case(*c, storage=storage, math_mode=math_mode) for c in CASES]


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--math", default="exact", choices=["exact", "fast"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16dev", "f64"])
    ap.add_argument("--json", action="store_true")
    a = ap.parse_args()
    rows = run_all(a.storage, a.math)
    if a.json:
        print(json.dumps(rows))
        return
    print(f"{'case':12s} {'Cd':>7s} {'Cl':>7s} {'published':>12s} {'solid':>6s} {'A':>5s}")
    for r in rows:
        pub = ", ".join(f"{k}={v:+.2f}" for k, v in r["published"].items())
        print(f"{r['case']:12s} {r['cd']:7.3f} {r['cl']:7.3f} {pub:>12s} {r['solid_cells']:6d} "
              f"{r['area']:5d}")


if __name__ == "__main__":
    main()
