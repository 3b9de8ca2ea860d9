"""The CUDA step (exact arithmetic, through the C ABI) against the reference's own outputs.

Replays every golden case of tests/golden on the GPU with WT_MATH_EXACT and
float32 storage: all arrays must match the reference bit for bit; the force
series within 1e-12 relative (the GPU sums per-cell terms in a tree).
The fast float32 collision is held to the FAST_RTOL bound on the fields.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from test_oracle_golden import SOLVER_CASES, replay_and_compare

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def golden(wt_lib):
    return json.loads((GOLDEN / "golden.json").read_text()), np.load(GOLDEN / "golden.npz")


@pytest.mark.parametrize("name", SOLVER_CASES)
def test_gpu_exact_reproduces_reference(golden, name):
    from windtunnel_b200 import LBM
    manifest, arrays = golden
    entry = manifest["solver"][name]
    g = LBM(*entry["case"]["dims"], math="exact", kernel="direct")
    replay_and_compare(g, name, entry, arrays, 1e-12, lambda s, n: s.step_forces(n))
    want = entry["stats2"] if "stats2" in entry else entry["stats"]
    assert [g.frontalArea, g.planformArea, g.solidCells, g.rideHeight,
            bool(g.movingWalls)] == want
    pts = arrays[f"{name}.sample_pts"]
    assert np.array_equal(g.sample_points(pts), arrays[f"{name}.sample_out"])
    assert [int(g.isSolid(*p)) for p in pts] == arrays[f"{name}.is_solid"].tolist()


def test_gpu_lookup_reproduces_body_makeTest(golden):
    from windtunnel_b200 import LBM
    manifest, arrays = golden
    vox = manifest["voxel"]
    grid = arrays["mesh.grid"].reshape(vox["nz"], vox["ny"], vox["nx"])
    nx, ny, nz = manifest["lookup"]["dims"]
    for k, c in enumerate(manifest["lookup"]["cases"]):
        g = LBM(nx, ny, nz, math="exact")
        g.voxelize_grid(grid, vox["min"], vox["inv"], c["M"], c["P"], c["scale"], c["box"])
        assert np.array_equal(g.solid, arrays[f"lookup{k}.solid"]), k
        assert [g.frontalArea, g.planformArea, g.solidCells, g.rideHeight] == c["stats"]


@pytest.mark.parametrize("name", ["sphere", "ground_road_spin"])
def test_gpu_fast_close_to_reference(golden, name):
    from test_oracle_golden import replay_setup
    from windtunnel_b200 import LBM
    manifest, arrays = golden
    entry = manifest["solver"][name]
    g = LBM(*entry["case"]["dims"], math="fast")
    replay_setup(g, name, entry)
    last = entry["case"]["snaps"][-1]
    F = g.step_forces(last)
    want = arrays[f"{name}.forces"][:last]
    assert np.abs(F - want).max() <= 1e-4 * np.abs(want).max()
    if f"{name}.{last}.ux" in arrays.files:
        for k, a in zip(("ux", "uy", "uz"), g.fields()[:3]):
            ref = arrays[f"{name}.{last}.{k}"]
            assert np.abs(a - ref).max() <= 1e-5 * max(np.abs(ref).max(), 1e-3), k
