"""CPU checks of the oracle itself (no GPU): invariants the reference guarantees."""
import numpy as np
import pytest

from lbm_cases import apply_case


@pytest.fixture(scope="module")
def O(oracle_lib):
    return oracle_lib


def splitmix64_draw(seed: int, k: int) -> float:
    M = (1 << 64) - 1
    z = (seed + (k + 1) * 0x9E3779B97F4A7C15) & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    z ^= z >> 31
    return (z >> 11) * 2.0 ** -53


def test_splitmix64_stream(O):
    for seed in (0, 1234, 2 ** 63 + 17):
        for k in (0, 1, 2, 999, 10 ** 9):
            assert O.uniform_draw(seed, k) == splitmix64_draw(seed, k)


def test_toint32_matches_ecmascript(O):
    f = O.lib().or_toint32_export
    cases = {3.7: 3, -3.7: -3, -0.5: 0, 0.0: 0, 2.0 ** 31: -(2 ** 31), 2.0 ** 32 + 5: 5,
             -(2.0 ** 31) - 1: 2 ** 31 - 1, float("nan"): 0, float("inf"): 0, 1e20: 1661992960}
    for v, want in cases.items():
        assert f(v) == want, v


def test_voxel_range_clamps_like_reference(O):
    # js/lbm.js:216-218: floor/ceil then clamp to [1, n-2]
    assert O.voxel_range(20, 10, 10, [-5.5, 2.2, 3.0, 30.1, 7.9, 8.0]) == (1, 18, 2, 8, 3, 8)
    assert O.voxel_range(20, 10, 10, [5, 5, 5, 4, 4, 4]) == (5, 4, 5, 4, 5, 4)


@pytest.mark.parametrize("side_bc", ["eq", "freeslip"])
def test_uniform_flow_is_a_fixed_point(O, side_bc):
    o = O.OracleLBM(20, 12, 10, side_bc=side_bc)
    apply_case(o, side_bc=side_bc, amp=0)
    o.reset()
    o.step_forces(20)
    ux, uy, uz, rho = o.fields()
    tol = 0.0 if side_bc == "freeslip" else 1e-9
    assert np.abs(ux - np.float32(0.05)).max() <= tol
    assert np.abs(uy).max() <= tol and np.abs(uz).max() <= tol
    assert np.abs(rho - 1).max() <= tol


@pytest.mark.parametrize("threads", [2, 3, 5])
def test_pool_decomposition_is_bit_identical(O, threads):
    """js/pool.js splits z into slabs; fields and populations do not change (README.md:260-262)."""
    runs = []
    for t in (1, threads):
        o = O.OracleLBM(30, 14, 17)
        apply_case(o, sphere=(10.0, 7.0, 8.5, 3.5), ground=True, roadVel=0.04)
        F = o.step_forces(12, threads=t)
        runs.append((F, o.populations("f", "raw"), o.populations("g", "raw"), o.fields()))
    (F1, f1, g1, u1), (F2, f2, g2, u2) = runs
    assert np.array_equal(f1, f2) and np.array_equal(g1, g2)
    for a, b in zip(u1, u2):
        assert np.array_equal(a, b)
    assert np.abs(F1 - F2).max() <= 1e-12 * np.abs(F1).max()


def test_voxelize_statistics(O):
    o = O.OracleLBM(40, 20, 20)
    apply_case(o, sphere=(12.0, 10.0, 10.0, 4.0), amp=0)
    s = o.body_stats()
    solid = o.solid.reshape(20, 20, 40)
    assert s.solid_cells == int((solid == 1).sum())
    assert s.frontal_area == int((solid == 1).any(axis=2).sum())
    assert s.planform_area == int((solid == 1).any(axis=1).sum())
    # cell centres within r
    z, y, x = np.mgrid[0:20, 0:20, 0:40] + 0.5
    assert s.solid_cells == int(((x - 12) ** 2 + (y - 10) ** 2 + (z - 10) ** 2 <= 16).sum())
    near = o.near.reshape(20, 20, 40)
    assert near.sum() > 0 and not (near & (solid > 0)).any()


def test_equilibrium_state_has_reference_moments(O):
    o = O.OracleLBM(12, 8, 8, "f64")
    o.set_params(u0=0.07)
    o.reset()
    f = o.populations("f", "f64")
    W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    EX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
    rho = 1 + f.sum(axis=0)
    jx = (EX[:, None] * (f + W[:, None])).sum(axis=0)
    assert np.allclose(rho, 1, atol=1e-15)
    assert np.allclose(jx, 0.07, atol=1e-15)
