"""The oracle's discrete adjoint of the partial-bounce-back step (CPU).

The FP64 oracle's gradient dJ/ds, J the mean drag over the last steps of a
run, must equal central finite differences of the FP64 oracle's own forward
run. This pins the adjoint that the GPU kernels are compared with.
Central differences with eps = 1e-4 carry an O(eps^2) truncation error;
measured agreement is 1e-9..1.4e-6 relative; the bar is 2e-5.
"""
import numpy as np
import pytest

from lbm_cases import apply_case

FD_RTOL = 2e-5
DIMS = (20, 10, 10)
BOX = (5, 2, 2, 11, 8, 8)


def smoothed_sphere(box, centre, radius, width, noise, seed):
    """s = (1 - tanh((|x - c| - r) / w)) / 2 + U(-noise, noise), clipped to [0, 1]."""
    x0, y0, z0, x1, y1, z1 = box
    zz, yy, xx = np.meshgrid(np.arange(z0, z1) + 0.5, np.arange(y0, y1) + 0.5,
                             np.arange(x0, x1) + 0.5, indexing="ij")
    r = np.sqrt((xx - centre[0]) ** 2 + (yy - centre[1]) ** 2 + (zz - centre[2]) ** 2)
    rng = np.random.default_rng(seed)
    s = 0.5 * (1 - np.tanh((r - radius) / width)) + rng.uniform(-noise, noise, r.shape)
    return np.clip(s, 0.0, 1.0)


def _make(s, **kw):
    from oracle.oracle import OracleLBM
    o = OracleLBM(*DIMS, "f64", side_bc=kw.get("side_bc", "eq"))
    apply_case(o, u0=0.05, tau=0.53, **kw)
    o.set_solid_fraction(BOX, s)
    return o


CASES = {
    "trt-les": dict(),
    "freeslip": dict(side_bc="freeslip"),
    "les-off": dict(les=False),
    "bgk": dict(trt=False),
    "binary-body": dict(sphere=(15.0, 5.0, 5.0, 1.8)),
    "ground": dict(ground=True, side_bc="freeslip"),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_adjoint_matches_central_differences(oracle_lib, name):
    kw = CASES[name]
    s0 = smoothed_sphere(BOX, (8.0, 5.0, 5.0), 2.5, 1.0, 0.05, seed=5)
    N, W = 60, 20
    J, g = _make(s0, **kw).adjoint(N, W)
    fwd = _make(s0, **kw).step_forces(N)
    assert J == pytest.approx(fwd[-W:, 0].mean(), rel=1e-14)
    rng = np.random.default_rng(11)
    eps = 1e-4
    for _ in range(4):
        idx = tuple(int(rng.integers(0, n)) for n in s0.shape)
        sp, sm = s0.copy(), s0.copy()
        sp[idx] += eps
        sm[idx] -= eps
        jp = _make(sp, **kw).step_forces(N)[-W:, 0].mean()
        jm = _make(sm, **kw).step_forces(N)[-W:, 0].mean()
        fd = (jp - jm) / (2 * eps)
        assert abs(g[idx] - fd) <= FD_RTOL * max(abs(fd), 1e-3 * np.abs(g).max()), (idx, g[idx], fd)


def test_solid_fraction_zero_is_the_plain_step(oracle_lib):
    """s = 0 everywhere leaves the step bit-identical to a lattice without the field."""
    from oracle.oracle import OracleLBM
    a = OracleLBM(*DIMS, "f32")
    b = OracleLBM(*DIMS, "f32")
    for o in (a, b):
        apply_case(o, u0=0.05, tau=0.53, sphere=(9.0, 5.0, 5.0, 2.0))
    b.set_solid_fraction(BOX, np.zeros((6, 6, 6)))
    fa, fb = a.step_forces(12), b.step_forces(12)
    assert np.array_equal(fa, fb)
    assert np.array_equal(a.populations("f", "raw"), b.populations("f", "raw"))
