"""The host restatement of the reference's analytic bodies (js/shapes.js).

Each catalogue body placed as test.html:62-68 places it (fit, position,
pitch) must give the reference's own scale, rotation and occupancy (golden,
produced by the unmodified js/shapes.js + js/lbm.js) bit for bit.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def golden_bodies():
    m = json.loads((GOLDEN / "golden.json").read_text())["bodies"]
    return m, np.load(GOLDEN / "golden.npz")


def place(key, dims, ground, aoa):
    from windtunnel_b200.shapes import Body
    nx, ny, nz = dims
    b = Body(key)
    b.fit(nx, ny, nz)
    b.pos = [nx * 0.36, 1 if ground else ny * 0.5, nz * 0.5]
    b.pitch = -aoa * math.pi / 180
    return b


@pytest.mark.parametrize("key", ["sphere", "cube", "cylinder", "teardrop", "sedan", "truck",
                                 "wing", "airplane", "sports"])
def test_body_reproduces_reference_occupancy(oracle_lib, golden_bodies, key):
    m, arrays = golden_bodies
    c = m["cases"][key]
    b = place(key, m["dims"], c["ground"], c["aoa"])
    assert b.scale == c["scale"]
    assert b.M == c["M"]
    o = oracle_lib.OracleLBM(*m["dims"])
    o.voxelize(b.make_test(), b.box(), c["ground"])
    assert np.array_equal(o.solid, arrays[f"body.{key}.solid"])
    s = o.body_stats()
    assert [s.frontal_area, s.planform_area, s.solid_cells, s.ride_height] == c["stats"]
