"""Voxel.build (js/voxel.js:48-232): the oracle and the GPU build.

* The oracle's restatement reproduces the reference's own grid (golden,
  produced by the unmodified js/voxel.js) bit for bit, with its cell size,
  min corner and statistics.
* The GPU build (wt_voxel_build) reproduces the golden grid and the oracle's
  grid bit for bit, on the golden mesh at several resolutions and on the
  benchmark's 20000-triangle hull.
* The reference's own conservative bounds (testmodels.html:137-162): a
  watertight mesh has openness < 0.02 and encloses at least the voxel count
  of its analytic volume's interior.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def golden_mesh():
    m = json.loads((GOLDEN / "golden.json").read_text())["voxel"]
    a = np.load(GOLDEN / "golden.npz")
    return a["mesh.P"], a["mesh.grid"], m


def test_oracle_voxel_build_reproduces_reference(oracle_lib, golden_mesh):
    from oracle.oracle import voxel_build
    P, grid, m = golden_mesh
    g, info = voxel_build(P, m["res"])
    assert (info["nx"], info["ny"], info["nz"]) == (m["nx"], m["ny"], m["nz"])
    assert info["cell"] == m["cell"] and info["inv"] == m["inv"] and info["min"] == m["min"]
    assert info["solid"] == m["solid"] and info["openness"] == m["openness"]
    assert hashlib.sha256(g.tobytes()).hexdigest() == m["grid_sha256"]
    assert np.array_equal(g.ravel(), grid)


def test_hull_mesh_is_closed_and_oriented():
    from windtunnel_b200.mesh import hull_mesh, orient
    P = hull_mesh()
    assert P.dtype == np.float32 and P.size == 9 * 20000
    k = orient(P, 0, 1)
    V = P.reshape(-1, 3).astype(np.float64)
    assert V[:, 0].max() - V[:, 0].min() == pytest.approx(1.0, abs=1e-6)
    assert k > 0
    # every edge is shared by exactly two triangles (closed surface), poles aside
    T = P.reshape(-1, 3, 3)
    keys = {}
    for t in T:
        v = [tuple(x) for x in t]
        if len(set(v)) < 3:
            continue   # zero-area triangle of a pole fan
        for a, b in ((0, 1), (1, 2), (2, 0)):
            e = tuple(sorted((v[a], v[b])))
            keys[e] = keys.get(e, 0) + 1
    assert set(keys.values()) == {2}


def test_oracle_hull_is_watertight(oracle_lib):
    from oracle.oracle import voxel_build
    from windtunnel_b200.mesh import hull_mesh, orient
    P = hull_mesh(nu=40, nv=40)
    orient(P, 0, 1)
    g, info = voxel_build(P, 64)
    assert info["openness"] < 0.02
    assert info["solid"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("res", [22, 9, 40, 96])
def test_gpu_voxel_build_matches_reference_and_oracle(wt_lib, oracle_lib, golden_mesh, res):
    from oracle.oracle import voxel_build as oracle_build
    from windtunnel_b200.mesh import voxel_build
    P, grid, m = golden_mesh
    v = voxel_build(P, res)
    g, info = oracle_build(P, res)
    assert np.array_equal(v.grid, g)
    assert (v.nx, v.ny, v.nz, v.solid) == (info["nx"], info["ny"], info["nz"], info["solid"])
    assert v.openness == info["openness"] and v.cell == info["cell"] and v.min == info["min"]
    if res == m["res"]:
        assert hashlib.sha256(v.grid.tobytes()).hexdigest() == m["grid_sha256"]


@pytest.mark.gpu
def test_gpu_voxel_build_of_the_benchmark_hull(wt_lib, oracle_lib):
    from oracle.oracle import voxel_build as oracle_build
    from windtunnel_b200.mesh import hull_mesh, orient, voxel_build
    P = hull_mesh()
    orient(P, 0, 1)
    v = voxel_build(P, 160)
    g, info = oracle_build(P, 160)
    assert np.array_equal(v.grid, g)
    assert v.solid == info["solid"] and v.openness == info["openness"]
    assert v.openness < 0.02
    assert v.tris == 20000


@pytest.mark.gpu
def test_gpu_voxel_build_errors(wt_lib):
    from windtunnel_b200 import WTError
    from windtunnel_b200.mesh import voxel_build
    with pytest.raises(WTError, match="no triangles"):
        voxel_build(np.zeros(0, np.float32), 32)
    with pytest.raises(WTError, match="degenerate"):
        voxel_build(np.ones(9, np.float32), 32)
