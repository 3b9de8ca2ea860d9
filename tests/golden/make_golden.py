"""Generate the golden vectors of tests/golden by running the reference itself.

    python tests/golden/make_golden.py --reference /path/to/windtunnel

(or set WT_REFERENCE_ROOT instead of passing --reference).

The unmodified js/lbm.js, js/voxel.js and js/shapes.js of the reference are
executed through tests/golden/jsmini.py (a JavaScript-subset engine; no JS
engine exists on this machine). Each case drives the reference's own public
interface (new LBM, voxelize, step, force, fields, f/g buffers, sample,
isSolid, Voxel.build, Shapes.Body.makeTest/box) on a small seeded input and
records what it produced: full arrays for the smallest snapshots, SHA-256
digests of the raw bytes for the rest. The seeded initial velocity noise is
applied through the reference's own LBM._writeEq (the reference has no
noise API). Output: golden.npz + golden.json next to this script.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import jsmini  # noqa: E402


def splitmix64_draw(seed: int, k: int) -> float:
    M = (1 << 64) - 1
    z = (seed + (k + 1) * 0x9E3779B97F4A7C15) & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    z ^= z >> 31
    return (z >> 11) * 2.0 ** -53


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load(ref: Path):
    src = [(ref / "js" / n).read_text() for n in ("lbm.js", "voxel.js", "shapes.js")]
    return jsmini.run(src)


# ---------------------------------------------------------------------------- set-up helpers
def sphere_inside(cx, cy, cz, r):
    r2 = r * r

    def inside(x, y, z, *_):
        dx, dy, dz = x - cx, y - cy, z - cz
        return dx * dx + dy * dy + dz * dz <= r2
    return inside


def box_inside(lo, hi):
    def inside(x, y, z, *_):
        return lo[0] <= x <= hi[0] and lo[1] <= y <= hi[1] and lo[2] <= z <= hi[2]
    return inside


def spin_wallvel(cx, cy, omega):
    def wall(x, y, z, out, *_):
        out[0] = -omega * (y - cy)
        out[1] = omega * (x - cx)
        out[2] = 0.0
        return True
    return wall


def jbox(b):
    return jsmini.JSObject(x0=b[0], y0=b[1], z0=b[2], x1=b[3], y1=b[4], z1=b[5])


def seed_noise(sim, seed, amp):
    """reset(), then equilibrium at u0 + noise on every fluid cell via LBM._writeEq."""
    sim.reset()
    for i in range(sim.n):
        if sim.solid[i]:
            continue
        vx = sim.u0 + amp * (2 * splitmix64_draw(seed, 3 * i) - 1)
        vy = amp * (2 * splitmix64_draw(seed, 3 * i + 1) - 1)
        vz = amp * (2 * splitmix64_draw(seed, 3 * i + 2) - 1)
        sim._writeEq(sim.f, i, 1, vx, vy, vz)
        sim._writeEq(sim.g, i, 1, vx, vy, vz)
        sim.ux[i] = vx
        sim.uy[i] = vy
        sim.uz[i] = vz
        sim.rho[i] = 1


def snapshot(sim):
    f32 = lambda a: np.frombuffer(a.tobytes(), np.float32).copy()
    return {
        "f": f32(sim.f), "g": f32(sim.g),
        "ux": f32(sim.ux), "uy": f32(sim.uy), "uz": f32(sim.uz), "rho": f32(sim.rho),
        "solid": np.frombuffer(sim.solid.tobytes(), np.uint8).copy(),
        "near": np.frombuffer(sim.near.tobytes(), np.uint8).copy(),
    }


# ---------------------------------------------------------------------------- solver cases
SOLVER_CASES = [
    dict(name="sphere", dims=(16, 10, 10), params=dict(u0=0.05, tau=0.512, csm=0.1, lam=3 / 16),
         body=("sphere", 6.0, 5.0, 5.0, 2.6), noise=(1234, 1e-4), snaps=(1, 4, 10), full=(10,)),
    dict(name="ground_road_spin", dims=(18, 10, 10),
         params=dict(u0=0.05, tau=0.512, csm=0.1, lam=3 / 16),
         body=("sphere", 7.0, 4.5, 5.0, 2.2), ground=True, road=0.04, spin=0.01,
         noise=(77, 2e-4), snaps=(3, 8)),
    dict(name="bgk_les_off", dims=(14, 9, 8),
         params=dict(u0=0.04, tau=0.52, csm=0.1, lam=3 / 16, trt=False, les=False),
         body=("sphere", 5.5, 4.5, 4.0, 2.0), noise=(5, 1e-4), snaps=(2, 6)),
    dict(name="defaults_box", dims=(15, 9, 9), params=None,
         body=("box", (4.2, 3.1, 3.3), (7.6, 5.9, 5.4)), noise=None, snaps=(1, 6)),
    dict(name="body_at_outlet", dims=(13, 9, 9), params=dict(u0=0.05, tau=0.512, csm=0.1,
                                                             lam=3 / 16),
         body=("sphere", 10.6, 4.5, 4.5, 2.3), noise=(9, 1e-4), snaps=(5,)),
    dict(name="revoxelize", dims=(16, 10, 10), params=dict(u0=0.05, tau=0.512, csm=0.1,
                                                          lam=3 / 16),
         body=("sphere", 6.0, 5.0, 5.0, 2.6), noise=(1234, 1e-4), snaps=(4,),
         move=(("sphere", 8.3, 4.6, 5.2, 2.4), True), after=(4,)),
]


def body_args(body):
    if body[0] == "sphere":
        _, cx, cy, cz, r = body
        return sphere_inside(cx, cy, cz, r), (cx - r - 2, cy - r - 2, cz - r - 2,
                                              cx + r + 2, cy + r + 2, cz + r + 2)
    _, lo, hi = body
    return box_inside(lo, hi), (lo[0] - 1, lo[1] - 1, lo[2] - 1, hi[0] + 1, hi[1] + 1, hi[2] + 1)


def run_solver_case(G, case, arrays, manifest):
    LBM = G.LBM
    sim = LBM(*case["dims"])
    p = case.get("params")
    if p:
        sim.u0, sim.tau, sim.csm, sim.lambda_ = p["u0"], p["tau"], p["csm"], p["lam"]
        if "trt" in p:
            sim.trt = p["trt"]
        if "les" in p:
            sim.les = p["les"]
    inside, box = body_args(case["body"])
    wall = None
    if case.get("spin"):
        b = case["body"]
        wall = spin_wallvel(b[1], b[2], case["spin"])
    sim.voxelize(inside, jbox(box), case.get("ground", False), wall, case.get("road", 0))
    if case.get("noise"):
        seed_noise(sim, *case["noise"])
    entry = {"case": {k: v for k, v in case.items() if k != "name"}, "box": box,
             "stats": [sim.frontalArea, sim.planformArea, sim.solidCells, sim.rideHeight,
                       bool(sim.movingWalls)], "snaps": []}
    forces = []

    def record(tag):
        s = snapshot(sim)
        digests = {k: sha(v) for k, v in s.items()}
        snap = {"tag": tag, "steps": sim.steps, "parity": sim.parity, "sha256": digests}
        if isinstance(tag, int) and tag in case.get("full", ()):
            for k, v in s.items():
                arrays[f"{case['name']}.{tag}.{k}"] = v
            snap["full"] = True
        entry["snaps"].append(snap)

    record("init")
    done = 0
    for target in case["snaps"]:
        while done < target:
            sim.step()
            forces.append(list(sim.force))
            done += 1
        record(target)
    if case.get("move"):
        inside2, box2 = body_args(case["move"][0])
        sim.voxelize(inside2, jbox(box2), case["move"][1], None, 0)
        entry["box2"] = box2
        entry["stats2"] = [sim.frontalArea, sim.planformArea, sim.solidCells, sim.rideHeight,
                           bool(sim.movingWalls)]
        record("moved")
        for _ in range(case["after"][0]):
            sim.step()
            forces.append(list(sim.force))
        record("after")
    arrays[f"{case['name']}.forces"] = np.array(forces, np.float64)
    # sampling after the run
    rng = np.random.default_rng(11)
    pts = rng.uniform(-1.0, 1.0, size=(40, 3)) * np.array(case["dims"]) * 0.6 + \
        np.array(case["dims"]) * 0.5
    out = jsmini.JSArray([0.0, 0.0, 0.0])
    samples = []
    for x, y, z in pts:
        sim.sample(float(x), float(y), float(z), out)
        samples.append(list(out))
    arrays[f"{case['name']}.sample_pts"] = pts
    arrays[f"{case['name']}.sample_out"] = np.array(samples, np.float64)
    arrays[f"{case['name']}.is_solid"] = np.array(
        [bool(sim.isSolid(float(x), float(y), float(z))) for x, y, z in pts], np.uint8)
    manifest["solver"][case["name"]] = entry


# ---------------------------------------------------------------------------- geometry cases
def bumpy_ellipsoid_mesh(nu=14, nv=10, semi=(1.0, 0.45, 0.35), seed=3):
    """A closed triangle soup: a seeded bumpy ellipsoid as a (u, v) grid."""
    rng = np.random.default_rng(seed)
    verts = []
    for j in range(nv + 1):
        th = math.pi * j / nv
        row = []
        for i in range(nu):
            ph = 2 * math.pi * i / nu
            bump = 1 + 0.08 * rng.standard_normal() if 0 < j < nv else 1.0
            row.append((semi[0] * bump * math.cos(th),
                        semi[1] * bump * math.sin(th) * math.cos(ph),
                        semi[2] * bump * math.sin(th) * math.sin(ph)))
        verts.append(row)
    tris = []
    for j in range(nv):
        for i in range(nu):
            a, b = verts[j][i], verts[j][(i + 1) % nu]
            c, d = verts[j + 1][i], verts[j + 1][(i + 1) % nu]
            if j > 0:
                tris.append((a, c, b))
            if j < nv - 1:
                tris.append((b, c, d))
    return np.array(tris, np.float32).reshape(-1)


def run_geometry_cases(G, arrays, manifest):
    Voxel, Shapes, LBM = G.Voxel, G.Shapes, G.LBM
    P = bumpy_ellipsoid_mesh()
    arrays["mesh.P"] = P
    Pj = jsmini.Float32Array(P.tolist())
    vox = Voxel.build(Pj, 22)
    grid = np.frombuffer(vox.grid.tobytes(), np.uint8).copy()
    arrays["mesh.grid"] = grid
    manifest["voxel"] = {"res": 22, "nx": vox.nx, "ny": vox.ny, "nz": vox.nz, "cell": vox.cell,
                         "min": list(vox.min), "inv": vox.inv, "ext": list(vox.ext),
                         "solid": vox.stats.solid, "openness": vox.stats.openness,
                         "tris": vox.stats.tris, "grid_sha256": sha(grid)}
    # the voxel-backed body placed by Body.makeTest / Body.box (js/shapes.js:353-388, :473-486)
    Shapes.BODIES["golden_mesh"] = jsmini.JSObject(
        name="golden", ground=False, custom=True, fill=0.7, parts=jsmini.JSArray(), vox=vox)
    lookups = []
    for k, (yaw, pitch, scale, pos) in enumerate([(0.3, -0.1, 7.0, (9.3, 7.1, 6.8)),
                                                   (math.radians(15), 0.0, 9.5, (10.0, 7.0, 7.0)),
                                                   (-1.1, 0.4, 6.2, (11.6, 6.4, 7.7))]):
        b = Shapes.Body("golden_mesh")
        b.scale, b.yaw, b.pitch = scale, yaw, pitch
        b.pos = jsmini.JSArray(list(pos))
        test = b.makeTest()
        box = b.box()
        sim = LBM(24, 14, 14)
        sim.voxelize(test, box, False)
        solid = np.frombuffer(sim.solid.tobytes(), np.uint8).copy()
        arrays[f"lookup{k}.solid"] = solid
        lookups.append({"M": list(b.M), "P": list(pos), "scale": scale,
                        "box": [box.x0, box.y0, box.z0, box.x1, box.y1, box.z1],
                        "stats": [sim.frontalArea, sim.planformArea, sim.solidCells,
                                  sim.rideHeight]})
    manifest["lookup"] = {"dims": [24, 14, 14], "cases": lookups}
    # analytic catalogue occupancy, placed as test.html:62-68 does
    bodies = {}
    for key, ground, aoa in [("sphere", False, 0), ("cube", False, 0), ("cylinder", False, 0),
                             ("teardrop", False, 0), ("sedan", True, 0), ("truck", True, 0),
                             ("wing", False, 8), ("airplane", False, 2), ("sports", True, 0)]:
        NX, NY, NZ = 48, 22, 22
        b = Shapes.Body(key)
        b.fit(NX, NY, NZ)
        b.pos = jsmini.JSArray([NX * 0.36, 1 if ground else NY * 0.5, NZ * 0.5])
        b.pitch = -aoa * math.pi / 180
        sim = LBM(NX, NY, NZ)
        sim.voxelize(b.makeTest(), b.box(), ground)
        solid = np.frombuffer(sim.solid.tobytes(), np.uint8).copy()
        arrays[f"body.{key}.solid"] = solid
        bodies[key] = {"ground": ground, "aoa": aoa, "scale": b.scale, "M": list(b.M),
                       "stats": [sim.frontalArea, sim.planformArea, sim.solidCells,
                                 sim.rideHeight]}
    manifest["bodies"] = {"dims": [48, 22, 22], "cases": bodies}


def generate(ref: Path) -> tuple[dict, dict]:
    """Run every case through the reference checkout at `ref`: (manifest, arrays)."""
    G = load(ref)
    arrays: dict = {}
    manifest = {"generator": "tests/golden/make_golden.py (reference js/ run through jsmini)",
                "solver": {}}
    for case in SOLVER_CASES:
        run_solver_case(G, case, arrays, manifest)
    run_geometry_cases(G, arrays, manifest)
    return manifest, arrays


def main():
    import os
    ap = argparse.ArgumentParser()
    env = os.environ.get("WT_REFERENCE_ROOT")
    ap.add_argument("--reference", type=Path, required=env is None,
                    default=Path(env) if env else None,
                    help="root of the windtunnel checkout (holds js/lbm.js); "
                         "default: $WT_REFERENCE_ROOT")
    a = ap.parse_args()
    manifest, arrays = generate(a.reference)
    np.savez_compressed(HERE / "golden.npz", **arrays)
    (HERE / "golden.json").write_text(json.dumps(manifest, indent=1, default=float))
    print("wrote", HERE / "golden.npz", (HERE / "golden.npz").stat().st_size, "bytes")


if __name__ == "__main__":
    main()
