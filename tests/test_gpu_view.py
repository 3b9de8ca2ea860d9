"""The flow-visualisation arithmetic on the GPU (js/main.js:691-709, :925-968).

wt_slice and wt_advect against a float64 numpy restatement over the
lattice's own fields: the slice scalars to 1e-6 relative (float32 output),
the particle positions exactly as LBM.sample moves them.
"""
import numpy as np
import pytest

from lbm_cases import apply_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sim(wt_lib):
    from windtunnel_b200 import LBM
    s = LBM(40, 20, 18)
    apply_case(s, sphere=(14.0, 10.0, 9.0, 4.0))
    s.step_forces(60)
    return s


def _expected(sim, plane, k, field):
    nx, ny, nz = sim.nx, sim.ny, sim.nz
    ux, uy, uz, rho = (a.astype(np.float64).reshape(nz, ny, nx) for a in sim.fields())
    solid = sim.solid.reshape(nz, ny, nx) != 0
    u0 = sim.u0
    if plane == "xy":
        U, V, W, R, S = ux[k], uy[k], uz[k], rho[k], solid[k]
    else:
        U, V, W, R, S = ux[:, k], uy[:, k], uz[:, k], rho[:, k], solid[:, k]

    def nb(A):
        ip = np.concatenate([A[:, 1:], A[:, -1:]], axis=1)
        im = np.concatenate([A[:, :1], A[:, :-1]], axis=1)
        jp = np.concatenate([A[1:], A[-1:]], axis=0)
        jm = np.concatenate([A[:1], A[:-1]], axis=0)
        return ip, im, jp, jm
    if field == "speed":
        t = np.sqrt(U * U + V * V + W * W) / u0
    elif field == "pressure":
        ip, im, jp, jm = nb(R)
        r = (R * 2 + ip + im + jp + jm) / 6
        t = ((r - 1) / 3) / (0.5 * u0 * u0)
    else:
        if plane == "xy":
            vip, vim, _, _ = nb(V)
            _, _, ujp, ujm = nb(U)
            w = (vip - vim) * 0.5 - (ujp - ujm) * 0.5
        else:
            _, _, ujp, ujm = nb(U)
            wip, wim, _, _ = nb(W)
            w = (ujp - ujm) * 0.5 - (wip - wim) * 0.5
        t = w / u0
    return np.where(S, np.nan, t).astype(np.float32)


@pytest.mark.parametrize("plane,k", [("xy", 9), ("xz", 10)])
@pytest.mark.parametrize("field", ["speed", "pressure", "vorticity"])
def test_slice_matches_restatement(sim, plane, k, field):
    got = sim.slice(plane, k, field)
    want = _expected(sim, plane, k, field)
    assert np.array_equal(np.isnan(got), np.isnan(want))
    m = ~np.isnan(want)
    assert np.all(np.abs(got[m] - want[m]) <= 1e-6 * np.maximum(np.abs(want[m]), 1e-3))
    if plane == "xy":
        assert np.isnan(got).sum() > 0      # the sphere cuts the plane


def test_advect_moves_particles_by_the_sampled_velocity(sim):
    rng = np.random.default_rng(2)
    p0 = rng.uniform([1, 1, 1], [39, 19, 17], size=(300, 3))
    v = sim.sample_points(p0)
    k = 2.5
    p1, expired, speed = sim.advect(p0, k)
    assert np.array_equal(p1, p0 + v * k)
    assert np.allclose(speed, np.sqrt((v ** 2).sum(1)) / sim.u0, rtol=1e-6)
    nx, ny, nz = sim.nx, sim.ny, sim.nz
    out = ((p1[:, 0] > nx - 2) | (p1[:, 0] < 0.5) | (p1[:, 1] < 0.8) | (p1[:, 1] > ny - 1.2) |
           (p1[:, 2] < 0.8) | (p1[:, 2] > nz - 1.2) |
           np.array([sim.isSolid(*p) for p in p1]))
    assert np.array_equal(expired, out)
