"""The reference's validation page (test.html) on the GPU path.

* With the exact arithmetic and float32 storage the GPU step is the
  reference's: on the test.html runs the drag and lift coefficients equal
  those of the CPU oracle (the bit-exact restatement of js/lbm.js) to 1e-9
  relative (the force sums run in a different order).
* The bluff-body drag also lies within 0.015 of the values the reference's
  README publishes for these runs (printed to two decimals). Its wing-lift
  values are not reproduced by the reference's current code either -- the
  oracle, pinned to the unmodified js/lbm.js, gives Cl = 0.315 at +8 degrees
  where the README lists 0.42 -- so the wing is held to test.html's own
  colouring: the lift follows the sign of the angle of attack.
* The fast float32 collision stays within 2% of the exact one, or within
  the sampling noise of the unsteady wakes' 300-step means where that is
  larger.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BLUFF = ("sphere", "cube", "cylinder", "teardrop", "sedan", "truck")


@pytest.fixture(scope="module")
def exact_rows(wt_lib):
    from windtunnel_b200.validate import run_all
    return {r["case"]: r for r in run_all("f32", "exact")}


def _oracle_case(name):
    from oracle.oracle import OracleLBM
    from windtunnel_b200.shapes import Body
    from windtunnel_b200.validate import AVG, CASES, NX, NY, NZ, TAU, WARM
    _, key, ground, aoa = next(c for c in CASES if c[0] == name)
    o = OracleLBM(NX, NY, NZ, "f32")
    o.set_params(tau=TAU)
    b = Body(key)
    b.fit(NX, NY, NZ)
    b.pos = [NX * 0.36, 1 if ground else NY * 0.5, NZ * 0.5]
    b.pitch = -aoa * math.pi / 180
    o.voxelize(b.make_test(), b.box(), ground)
    s = o.body_stats()
    area = s.planform_area if b.ref == "planform" else s.frontal_area
    o.step_forces(WARM, threads=8)
    F = o.step_forces(AVG, threads=8)
    q = 0.5 * o.params().u0 ** 2 * area
    return F[:, 0].mean() / q, F[:, 1].mean() / q


@pytest.mark.parametrize("name", ["sphere", "sedan", "wing a=8"])
def test_validation_equals_the_reference_arithmetic(oracle_lib, exact_rows, name):
    cd, cl = _oracle_case(name)
    r = exact_rows[name]
    assert r["cd"] == pytest.approx(cd, rel=1e-9)
    assert r["cl"] == pytest.approx(cl, rel=1e-9, abs=1e-12)


def test_bluff_body_drag_near_published_values(exact_rows):
    for name in BLUFF:
        r = exact_rows[name]
        assert abs(r["cd"] - r["published"]["cd"]) <= 0.015, (name, r["cd"])


def test_validation_signs_as_test_html_colours_them(exact_rows):
    """test.html:84-88: Cd > 0 everywhere, Cl follows the sign of the angle."""
    for name, r in exact_rows.items():
        assert r["cd"] > 0, name
    assert exact_rows["wing a=8"]["cl"] > 0 and exact_rows["wing a=-8"]["cl"] < 0
    assert exact_rows["wing a=16"]["cl"] > exact_rows["wing a=8"]["cl"]


def test_fast_collision_close_to_exact(exact_rows):
    """At the page's viscosity (tau - 1/2 = 3e-3) the wakes are unsteady, so
    two arithmetic forms follow different trajectories after a few hundred
    steps: the 300-step mean drags agree to 2% or to three combined blocking
    standard errors of those means, whichever is larger."""
    from windtunnel_b200.validate import CASES, run_case
    for c in CASES[:6]:
        r = run_case(*c, storage="f32", math_mode="fast")
        e = exact_rows[c[0]]
        tol = max(0.02 * abs(e["cd"]), 3 * math.hypot(r["cd_sem"], e["cd_sem"]))
        assert abs(r["cd"] - e["cd"]) <= tol, (c[0], r["cd"], e["cd"], tol)
