"""The oracle against golden vectors produced by the reference itself.

tests/golden/golden.{npz,json} were made by tests/golden/make_golden.py, which
runs the unmodified js/lbm.js, js/voxel.js and js/shapes.js through a
JavaScript-subset engine. Every case is replayed here on the CPU oracle and
must agree bit for bit: populations (both buffers), fields, occupancy, near
flags, body statistics, the per-step force series (the single-thread oracle
sums forces in the reference's order), samples and the occupancy lookup.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def golden():
    manifest = json.loads((GOLDEN / "golden.json").read_text())
    arrays = np.load(GOLDEN / "golden.npz")
    return manifest, arrays


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def replay_setup(sim, name, entry):
    """Configure a simulator (oracle or GPU mirror) exactly as the golden case was."""
    from lbm_cases import spinning_sphere_wallvel
    from windtunnel_b200.lbm import sphere_inside
    case = entry["case"]
    p = case.get("params")
    if p:
        kw = dict(u0=p["u0"], tau=p["tau"], csm=p["csm"], trt=int(p.get("trt", True)),
                  les=int(p.get("les", True)))
        kw["lambda"] = p["lam"]
        sim.set_params(**kw)
    body = case["body"]
    if body[0] == "sphere":
        inside = sphere_inside(*body[1:5])
    else:
        lo, hi = body[1], body[2]

        def inside(x, y, z):
            return ((lo[0] <= x) & (x <= hi[0]) & (lo[1] <= y) & (y <= hi[1]) &
                    (lo[2] <= z) & (z <= hi[2]))
    wall = None
    if case.get("spin"):
        # the same closure as the golden generator's spin_wallvel
        cx, cy, om = body[1], body[2], case["spin"]

        def wall(x, y, z, out):
            out[0] = -om * (y - cy)
            out[1] = om * (x - cx)
            out[2] = 0.0
            return True
    sim.voxelize(inside, entry["box"], case.get("ground", False), wall, case.get("road", 0))
    if case.get("noise"):
        sim.init_eq_noise(*case["noise"])


def snapshot_digests(sim):
    f = sim.populations("f", "raw")
    g = sim.populations("g", "raw")
    ux, uy, uz, rho = sim.fields()
    parts = {"f": f, "g": g, "ux": ux, "uy": uy, "uz": uz, "rho": rho,
             "solid": sim.solid, "near": sim.near}
    return {k: sha(v) for k, v in parts.items()}, parts


def replay_and_compare(sim, name, entry, arrays, force_rtol, stepper):
    """Run the case on sim; compare every snapshot; returns the force series."""
    from windtunnel_b200.lbm import sphere_box, sphere_inside
    replay_setup(sim, name, entry)
    case = entry["case"]
    forces = []
    done = 0
    for snap in entry["snaps"]:
        tag = snap["tag"]
        if tag == "moved":
            b = case["move"][0]
            sim.voxelize(sphere_inside(*b[1:5]), entry["box2"], case["move"][1], None, 0)
        elif tag == "after":
            forces.append(stepper(sim, case["after"][0]))
        elif tag != "init":
            forces.append(stepper(sim, tag - done))
            done = tag
        digests, parts = snapshot_digests(sim)
        bad = [k for k in digests if digests[k] != snap["sha256"][k]]
        if bad and snap.get("full"):
            for k in bad:
                ref = arrays[f"{name}.{tag}.{k}"]
                diff = np.flatnonzero(ref.reshape(-1) != parts[k].reshape(-1))
                print(name, tag, k, "differs at", diff[:10])
        assert not bad, f"{name} @ {tag}: {bad} differ from the reference"
    got = np.concatenate(forces)
    want = arrays[f"{name}.forces"]
    assert got.shape == want.shape
    if force_rtol == 0:
        assert np.array_equal(got, want), np.abs(got - want).max()
    else:
        assert np.abs(got - want).max() <= force_rtol * max(np.abs(want).max(), 1e-300)
    return sim


SOLVER_CASES = ["sphere", "ground_road_spin", "bgk_les_off", "defaults_box", "body_at_outlet",
                "revoxelize"]


@pytest.mark.parametrize("name", SOLVER_CASES)
def test_oracle_reproduces_reference(oracle_lib, golden, name):
    manifest, arrays = golden
    entry = manifest["solver"][name]
    o = oracle_lib.OracleLBM(*entry["case"]["dims"])
    replay_and_compare(o, name, entry, arrays, 0.0, lambda s, n: s.step_forces(n))
    s = o.body_stats()
    want = entry["stats2"] if "stats2" in entry else entry["stats"]
    assert [s.frontal_area, s.planform_area, s.solid_cells, s.ride_height,
            bool(s.moving_walls)] == want
    pts = arrays[f"{name}.sample_pts"]
    got = np.array([o.sample(*p) for p in pts])
    assert np.array_equal(got, arrays[f"{name}.sample_out"])
    assert [int(o.isSolid(*p)) for p in pts] == arrays[f"{name}.is_solid"].tolist()


def test_oracle_lookup_reproduces_body_makeTest(oracle_lib, golden):
    """js/shapes.js:365-388 (voxel-backed makeTest) + voxelize, on three placements."""
    manifest, arrays = golden
    vox = manifest["voxel"]
    grid = arrays["mesh.grid"].reshape(vox["nz"], vox["ny"], vox["nx"])
    nx, ny, nz = manifest["lookup"]["dims"]
    for k, c in enumerate(manifest["lookup"]["cases"]):
        mask = oracle_lib.lookup_mask(grid, vox["min"], vox["inv"], c["M"], c["P"], c["scale"],
                                      nx, ny, nz, c["box"])
        o = oracle_lib.OracleLBM(nx, ny, nz)
        o.voxelize_mask(c["box"], mask)
        assert np.array_equal(o.solid, arrays[f"lookup{k}.solid"]), k
        s = o.body_stats()
        assert [s.frontal_area, s.planform_area, s.solid_cells, s.ride_height] == c["stats"]


def test_golden_manifest_is_complete(golden):
    manifest, arrays = golden
    assert set(SOLVER_CASES) <= set(manifest["solver"])
    assert manifest["voxel"]["grid_sha256"] == sha(arrays["mesh.grid"])
    assert len(manifest["bodies"]["cases"]) == 9


def test_golden_comparison_detects_a_small_change(oracle_lib, golden):
    """A planted change in the oracle's input must break the digests.

    tau is raised by one part in 1e8 (below a float32 ulp of the populations'
    updates, far above a double ulp): enough to move some float32 roundings.
    """
    manifest, arrays = golden
    entry = json.loads(json.dumps(manifest["solver"]["sphere"]))
    entry["case"]["params"]["tau"] *= 1 + 1e-8
    o = oracle_lib.OracleLBM(*entry["case"]["dims"])
    with pytest.raises(AssertionError):
        replay_and_compare(o, "sphere", entry, arrays, 0.0, lambda s, n: s.step_forces(n))
