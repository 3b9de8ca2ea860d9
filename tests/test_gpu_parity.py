"""Parity of the CUDA step (through the C ABI) against the CPU oracle.

Bars:
  * WT_MATH_EXACT with float32 storage reproduces the reference arithmetic:
    populations (both buffers), fields, occupancy and near flags are
    bit-identical to the oracle; the per-step force agrees to 1e-12 relative
    (only the order of the global force sum differs).
  * float64 storage (the FP64 oracle form) is bit-identical to the float64
    oracle in the same way.
  * WT_MATH_FAST (float32 collision) stays within FAST_TOL (relative L-inf)
    of the oracle on u and rho after the stated number of steps.
"""
import numpy as np
import pytest

from lbm_cases import CFG0, apply_case, pair_average, rel_linf, spinning_sphere_wallvel

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-12   # exact mode: force summation order differs from the sequential sum
FAST_TOL = 2e-4      # fast float32 collision vs float64 reference arithmetic, u and rho


@pytest.fixture(scope="module")
def both(wt_lib, oracle_lib):
    from oracle.oracle import OracleLBM
    from windtunnel_b200 import LBM
    return LBM, OracleLBM


def make_pair(both, dims, storage="f32", math="exact", kernel="auto", **case):
    LBM, OracleLBM = both
    g = LBM(*dims, storage=storage, math=math, kernel=kernel)
    o = OracleLBM(*dims, storage="f64" if storage == "f64" else "f32")
    apply_case(g, **case)
    apply_case(o, **case)
    return g, o


def assert_force_close(fg, fo, rtol=FORCE_RTOL):
    fg, fo = np.asarray(fg), np.asarray(fo)
    scale = max(np.abs(fo).max(), 1e-300)
    assert np.abs(fg - fo).max() <= rtol * scale, (fg, fo)


def assert_bit_exact(g, o, raw_dtype):
    for which in ("f", "g"):
        a = g.populations(which, "raw")
        b = o.populations(which, "raw")
        assert a.dtype == np.dtype(raw_dtype)
        bad = np.flatnonzero(a.view(np.uint8) != b.view(np.uint8))
        assert bad.size == 0, f"{which}: {bad.size} bytes differ"
    for name, a, b in zip(("ux", "uy", "uz", "rho"), g.fields(), o.fields()):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
    assert np.array_equal(g.solid, o.solid)
    assert np.array_equal(g.near, o.near)


EXACT_CASES = {
    "sphere-default": dict(dims=(24, 12, 12), sphere=(8.0, 6.0, 6.0, 3.0)),
    "odd-dims-les-off": dict(dims=(33, 17, 13), sphere=(10.3, 8.1, 6.7, 4.2), les=False),
    "bgk": dict(dims=(24, 12, 12), sphere=(8.0, 6.0, 6.0, 3.0), trt=False),
    "lambda-quarter": dict(dims=(24, 12, 12), sphere=(8.0, 6.0, 6.0, 3.0), lam=0.25, tau=0.5035,
                           csm=0.14),
    "freeslip": dict(dims=(26, 14, 12), sphere=(9.0, 7.0, 6.0, 3.5), side_bc="freeslip"),
    "ground-rolling-road": dict(dims=(28, 14, 12), sphere=(9.0, 5.0, 6.0, 3.0), ground=True,
                                roadVel=0.05),
    "spinning-body": dict(dims=(24, 14, 12), sphere=(9.0, 7.0, 6.0, 3.5),
                          wallVel=spinning_sphere_wallvel(9.0, 7.0, 6.0, 0.01)),
    "body-at-outlet": dict(dims=(20, 12, 12), sphere=(17.5, 6.0, 6.0, 3.0)),
    "no-body": dict(dims=(16, 8, 8)),
}


EXACT_CASES["odd-shapes-freeslip"] = dict(dims=(40, 13, 11), sphere=(15.0, 6.5, 5.5, 3.6),
                                          side_bc="freeslip")
EXACT_CASES["long-rows-road"] = dict(dims=(136, 10, 9), sphere=(126.0, 5.0, 4.5, 3.2),
                                     ground=True, roadVel=0.03)


@pytest.mark.parametrize("name", sorted(EXACT_CASES))
def test_exact_f32_bit_identical(both, name):
    case = dict(EXACT_CASES[name])
    dims = case.pop("dims")
    g, o = make_pair(both, dims, "f32", "exact", **case)
    assert_bit_exact(g, o, np.float32)   # after voxelize + seeded init
    for nsteps in (1, 6, 23):
        fg = g.step_forces(nsteps)
        fo = o.step_forces(nsteps)
        assert_force_close(fg, fo)
        assert_bit_exact(g, o, np.float32)
    assert g.steps == o.steps == 30
    assert g.parity == o.parity


@pytest.mark.parametrize("name", ["sphere-default", "freeslip", "ground-rolling-road",
                                  "long-rows-road"])
def test_exact_f64_bit_identical(both, name):
    case = dict(EXACT_CASES[name])
    dims = case.pop("dims")
    g, o = make_pair(both, dims, "f64", "exact", **case)
    assert_bit_exact(g, o, np.float64)
    assert_force_close(g.step_forces(17), o.step_forces(17))
    assert_bit_exact(g, o, np.float64)


def test_exact_cfg0_shape_bit_identical(both):
    """The 128x64x64 sphere case for 40 steps, oracle on 8 threads (pool decomposition)."""
    c = CFG0
    g, o = make_pair(both, (c["nx"], c["ny"], c["nz"]), "f32", "exact",
                     u0=c["u0"], tau=c["tau"], csm=c["csm"], lam=c["lam"], sphere=c["sphere"],
                     side_bc="freeslip")
    fg = g.step_forces(40)
    fo = o.step_forces(40, threads=8)
    assert_force_close(fg, fo)
    assert_bit_exact(g, o, np.float32)


@pytest.mark.parametrize("kernel", ["direct", "lean", "pair"])
@pytest.mark.parametrize("side_bc", ["eq", "freeslip"])
def test_fast_f32_within_tolerance(both, side_bc, kernel):
    g, o = make_pair(both, (48, 24, 24), "f32", "fast", kernel=kernel,
                     sphere=(14.0, 12.0, 12.0, 5.0), side_bc=side_bc)
    fg = g.step_forces(200)
    fo = o.step_forces(200)
    gu = g.fields()
    ou = o.fields()
    for name, a, b in zip(("ux", "uy", "uz"), gu[:3], ou[:3]):
        assert rel_linf(a, b) < FAST_TOL, name
    assert np.abs(gu[3] - ou[3]).max() < FAST_TOL * 0.05   # rho-1 scale ~ 5e-2 of u0
    assert np.array_equal(g.solid, o.solid)
    # pair-averaged drag over the last 100 steps
    cg = pair_average(fg[:, 0])[-100:].mean()
    co = pair_average(fo[:, 0])[-100:].mean()
    assert abs(cg - co) <= 1e-3 * abs(co)


def test_fast_cfg0_drag_and_fields(both):
    """Config 0 (128x64x64 sphere, Re=200, TRT 3/16, Cs=0.1), fast FP32 vs the oracle.

    Pointwise after 200 steps (measured: 1.0e-6 relative on ux). The sphere
    wake turns unsteady, so pointwise trajectories of different roundings
    separate after ~700 steps -- the reference's own float32-storage run
    departs from float64 storage just as fast -- and after 2000 steps the
    pair-averaged Cd and Cl are compared instead.
    """
    c = CFG0
    dims = (c["nx"], c["ny"], c["nz"])
    g, o = make_pair(both, dims, "f32", "fast", u0=c["u0"], tau=c["tau"], csm=c["csm"],
                     lam=c["lam"], sphere=c["sphere"], side_bc="freeslip")
    fg = [g.step_forces(200)]
    fo = [o.step_forces(200, threads=8)]
    gu, ou = g.fields(), o.fields()
    for name, a, b in zip(("ux", "uy", "uz"), gu[:3], ou[:3]):
        assert rel_linf(a, b) < 1e-5, name
    fg.append(g.step_forces(1800))
    fo.append(o.step_forces(1800, threads=8))
    fg, fo = np.concatenate(fg), np.concatenate(fo)
    q = 0.5 * c["u0"] ** 2 * g.frontalArea
    cdg = pair_average(fg[:, 0])[-500:].mean() / q
    cdo = pair_average(fo[:, 0])[-500:].mean() / q
    clg = pair_average(fg[:, 1])[-500:].mean() / q
    clo = pair_average(fo[:, 1])[-500:].mean() / q
    assert abs(cdg - cdo) <= 1e-3 * abs(cdo), (cdg, cdo)
    assert abs(clg - clo) <= 1e-3 * abs(cdo), (clg, clo)


@pytest.mark.parametrize("kernel", ["direct", "lean", "pair"])
def test_f16dev_within_tolerance(both, kernel):
    g, o = make_pair(both, (48, 24, 24), "f16dev", "fast", kernel=kernel,
                     sphere=(14.0, 12.0, 12.0, 5.0))
    fg = g.step_forces(200)
    fo = o.step_forces(200)
    gu, ou = g.fields(), o.fields()
    assert rel_linf(gu[0], ou[0]) < 2e-2
    cg = pair_average(fg[:, 0])[-100:].mean()
    co = pair_average(fo[:, 0])[-100:].mean()
    assert abs(cg - co) <= 1e-2 * abs(co)


@pytest.mark.parametrize("math,kernel", [("fast", "direct"), ("fast", "lean"), ("fast", "pair"),
                                         ("exact", "direct")])
@pytest.mark.parametrize("side_bc", ["eq", "freeslip"])
def test_uniform_flow_is_preserved(both, math, kernel, side_bc):
    """A uniform stream past no body is a fixed point of the step (free-slip exactly)."""
    LBM, _ = both
    s = LBM(20, 12, 10, math=math, side_bc=side_bc, kernel=kernel)
    s.set_params(u0=0.05, tau=0.512)
    s.reset()
    s.step_forces(25)
    ux, uy, uz, rho = s.fields()
    tol = 0.0 if (side_bc == "freeslip" and math == "exact") else 1e-6
    assert np.abs(ux - np.float32(0.05)).max() <= tol * 0.05 + 1e-9
    assert np.abs(uy).max() <= tol and np.abs(uz).max() <= tol
    assert np.abs(rho - 1).max() <= tol


def test_batch_equals_single_steps(both):
    LBM, _ = both
    a = LBM(24, 12, 12, math="fast")
    b = LBM(24, 12, 12, math="fast")
    for s in (a, b):
        apply_case(s, sphere=(8.0, 6.0, 6.0, 3.0))
    fa = a.step_forces(40)
    fb = []
    for _ in range(40):
        b.step()
        fb.append(b.force)
    assert np.array_equal(fa, np.array(fb))
    assert np.array_equal(a.populations("f", "raw"), b.populations("f", "raw"))


@pytest.mark.parametrize("dims", [(64, 20, 18), (38, 12, 10), (130, 9, 9), (40, 11, 21),
                                  (136, 10, 9)])
@pytest.mark.parametrize("storage", ["f32", "f16dev"])
def test_kernels_agree(both, storage, dims):
    """The lean and direct kernels move the same values; the fast collision
    may round differently only where the two re-associate it differently."""
    LBM, _ = both
    nx = dims[0]
    sims = []
    for kernel in ("direct", "lean", "pair"):
        s = LBM(*dims, storage=storage, kernel=kernel, side_bc="freeslip")
        apply_case(s, sphere=(nx - 6.0, dims[1] / 2, dims[2] / 2, 3.1), side_bc="freeslip",
                   ground=True)
        sims.append((s.step_forces(30), s.fields(), s.populations("f", "f32")))
    fa, ua, pa = sims[0]
    for fb, ub, pb in sims[1:]:
        # half storage: a collision rounded differently may flip a half rounding (2^-11)
        assert np.abs(fa - fb).max() <= (1e-5 if storage == "f32" else 1e-3) * np.abs(fa).max()
        for a, b in zip(ua, ub):
            # half storage: one flipped half rounding moves u by ~5e-6; 30 steps compound it
            assert np.abs(a - b).max() <= (1e-6 if storage == "f32" else 2e-4)
        assert np.abs(pa - pb).max() <= (1e-6 if storage == "f32" else 1e-4)


@pytest.mark.parametrize("kernel,moving", [("lean", False), ("pair", False)])
@pytest.mark.parametrize("storage", ["f32", "f16dev"])
@pytest.mark.parametrize("side_bc", ["eq", "freeslip"])
def test_kernels_agree_with_direct_at_the_outlet(both, kernel, moving, storage, side_bc):
    """The lean and pair kernels against the direct kernel with the special
    rules they run: a body touching the outlet column, a road and the side
    planes; fields are checked on an intermediate and the last step."""
    LBM, _ = both
    dims = (40, 14, 12)
    out = []
    for kern in ("direct", kernel):
        s = LBM(*dims, storage=storage, kernel=kern, side_bc=side_bc)
        apply_case(s, sphere=(36.5, 6.0, 6.0, 3.4), side_bc=side_bc, ground=True,
                   roadVel=0.03 if moving else 0.0,
                   wallVel=spinning_sphere_wallvel(36.5, 6.0, 6.0, 0.01) if moving else None)
        f1 = s.step_forces(7)
        u1 = s.fields()
        f2 = s.step_forces(20)
        out.append((np.concatenate([f1, f2]), u1, s.fields(), s.populations("f", "f32")))
    (fa, ua1, ua2, pa), (fb, ub1, ub2, pb) = out
    assert np.abs(fa - fb).max() <= (1e-5 if storage == "f32" else 1e-3) * np.abs(fa).max()
    for a, b in list(zip(ua1, ub1)) + list(zip(ua2, ub2)):
        assert np.abs(a - b).max() <= (1e-6 if storage == "f32" else 2e-4)
    assert np.abs(pa - pb).max() <= (1e-6 if storage == "f32" else 1e-4)


@pytest.mark.parametrize("dims", [(40, 14, 12), (64, 20, 18), (130, 9, 9), (136, 10, 9),
                                  (4, 6, 6)])
@pytest.mark.parametrize("storage,rounding", [("f16dev", "nearest"), ("f16dev", "stochastic"),
                                              ("f32", "nearest")])
@pytest.mark.parametrize("side_bc", ["eq", "freeslip"])
def test_pair_kernel_agrees_with_lean(both, dims, storage, rounding, side_bc):
    """The pair kernel (two cells per thread, packed collision) against the
    lean kernel: a body touching the outlet column, a road, either side
    condition, rows of one, part of one and several 128-cell blocks and the
    smallest even row. Both collide in float32 with different
    re-associations, so the two agree to the half-storage tolerance of the
    other kernel comparisons (float32 storage: to the float32 one); the inlet
    column holds the equilibrium and the outlet column an exact copy of
    column nx-2 in both."""
    LBM, _ = both
    out = []
    nx, ny, nz = dims
    for kern in ("lean", "pair"):
        s = LBM(*dims, storage=storage, kernel=kern, side_bc=side_bc)
        if storage == "f16dev":
            s.set_params(f16_rounding=rounding)
        sphere = (nx - 4.5, ny / 2, nz / 2, 3.3) if nx > 8 else None
        apply_case(s, sphere=sphere, side_bc=side_bc, ground=True)
        f1 = s.step_forces(7)
        u1 = s.fields()
        f2 = s.step_forces(18)
        p = s.populations("f", "raw").reshape(19, nz, ny, nx)
        assert np.array_equal(p[:, 1:-1, 1:-1, -1], p[:, 1:-1, 1:-1, -2])
        out.append((np.concatenate([f1, f2]), u1, s.fields(), s.populations("f", "f32"),
                    p[:, 1:-1, 1:-1, 0].copy()))
    (fa, ua1, ua2, pa, ia), (fb, ub1, ub2, pb, ib) = out
    assert np.array_equal(ia, ib)        # inlet column: the equilibrium in both
    half = storage == "f16dev"
    scale = max(np.abs(fa).max(), 1e-30)
    assert np.abs(fa - fb).max() <= (1e-3 if half else 1e-5) * scale
    for a, b in list(zip(ua1, ub1)) + list(zip(ua2, ub2)):
        assert np.abs(a - b).max() <= (2e-4 if half else 1e-6)
    # stochastic rounding: the two kernels draw different random bits, so a
    # population may differ by a few half-precision steps after 25 steps
    assert np.abs(pa - pb).max() <= ((2e-4 if rounding == "stochastic" else 1e-4) if half else 1e-6)


def test_pair_kernel_conditions(both):
    from windtunnel_b200 import WTError
    from windtunnel_b200 import _lib as W
    LBM, _ = both
    for dims, storage, math in (((41, 12, 10), "f16dev", "fast"), ((41, 12, 10), "f32", "fast"),
                                ((40, 12, 10), "f32", "exact"), ((40, 12, 10), "f64", "exact")):
        s = LBM(*dims, storage=storage, math=math, kernel="pair")
        with pytest.raises(WTError) as e:
            s.step_forces(1)
        assert e.value.code == W.WT_ERR_UNSUPPORTED
    s = LBM(40, 12, 10, storage="f16dev", kernel="pair")
    apply_case(s, sphere=(20.0, 6.0, 5.0, 3.0), ground=True, roadVel=0.02)
    with pytest.raises(WTError):
        s.step_forces(1)
    # AUTO falls back to the direct kernel with moving walls, to lean for odd nx
    for dims, rv in (((40, 12, 10), 0.02), ((41, 12, 10), 0.0)):
        s = LBM(*dims, storage="f16dev")
        apply_case(s, sphere=(20.0, 6.0, 5.0, 3.0), ground=True, roadVel=rv)
        s.step_forces(3)


def test_lean_stochastic_rounding_agrees_with_direct(both):
    """Half storage with stochastic rounding: the lean kernel draws the direct
    kernel's random bits for the same cell and step, so the two agree to the
    half-storage tolerance of the other kernel comparisons, and the outlet
    column stays an exact copy of column nx-2."""
    LBM, _ = both
    dims = (40, 14, 12)
    out = []
    for kern in ("direct", "lean"):
        s = LBM(*dims, storage="f16dev", kernel=kern, side_bc="freeslip")
        s.set_params(f16_rounding="stochastic")
        apply_case(s, sphere=(20.0, 6.0, 6.0, 3.4), side_bc="freeslip", ground=True)
        f = s.step_forces(25)
        p = s.populations("f", "raw").reshape(19, dims[2], dims[1], dims[0])
        assert np.array_equal(p[:, 1:-1, 1:-1, -1], p[:, 1:-1, 1:-1, -2])
        out.append((f, s.fields(), s.populations("f", "f32")))
    (fa, ua, pa), (fb, ub, pb) = out
    assert np.abs(fa - fb).max() <= 1e-3 * np.abs(fa).max()
    for a, b in zip(ua, ub):
        assert np.abs(a - b).max() <= 2e-4
    assert np.abs(pa - pb).max() <= 1e-4


@pytest.mark.parametrize("kernel", ["lean", "pair"])
@pytest.mark.parametrize("storage", ["f32", "f16dev"])
def test_prefetch_changes_nothing(both, storage, kernel, monkeypatch):
    """The L2 prefetch distance of the lean and pair kernels (read at create
    time) moves timing only: off, the default and one past the end of the
    lattice give bit-identical populations and forces."""
    LBM, _ = both
    dims = (64, 20, 18)
    out = []
    for pf in ("0", None, str(64 * 20 * 18 * 2)):
        if pf is None:
            monkeypatch.delenv("WT_PREFETCH_CELLS", raising=False)
        else:
            monkeypatch.setenv("WT_PREFETCH_CELLS", pf)
        s = LBM(*dims, storage=storage, kernel=kernel, side_bc="freeslip")
        apply_case(s, sphere=(40.0, 10.0, 9.0, 4.2), side_bc="freeslip", ground=True)
        out.append((s.step_forces(25), s.populations("f", "raw")))
    monkeypatch.delenv("WT_PREFETCH_CELLS", raising=False)
    for f, p in out[1:]:
        assert np.array_equal(f, out[0][0])
        assert np.array_equal(p, out[0][1])


def test_step_is_deterministic(both):
    LBM, _ = both
    runs = []
    for _ in range(2):
        s = LBM(40, 20, 20, math="fast")
        apply_case(s, sphere=(12.0, 10.0, 10.0, 4.0))
        runs.append((s.step_forces(30), s.populations("f", "raw")))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


def test_voxelize_grid_matches_lookup(both):
    """Device evaluation of js/shapes.js:369-388 vs the oracle's, bit for bit."""
    from oracle.oracle import lookup_mask
    LBM, OracleLBM = both
    rng = np.random.default_rng(7)
    grid = (rng.random((9, 11, 17)) < 0.5).astype(np.uint8)   # (gnz, gny, gnx)
    gmin = [-0.61, -0.33, -0.27]
    ginv = 1 / 0.071
    yaw, pitch = 0.26, -0.11
    cy, sy, cp, sp = np.cos(yaw), np.sin(yaw), np.cos(pitch), np.sin(pitch)
    M = [cy * cp, -cy * sp, sy, sp, cp, 0.0, -sy * cp, sy * sp, cy]
    P = [14.3, 8.7, 9.1]
    scale = 11.5
    box = {"x0": 3.2, "y0": 1.1, "z0": 2.0, "x1": 25.9, "y1": 16.5, "z1": 16.2}
    g = LBM(30, 18, 18, math="exact")
    o = OracleLBM(30, 18, 18)
    g.voxelize_grid(grid, gmin, ginv, M, P, scale, box)
    mask = lookup_mask(grid, gmin, ginv, M, P, scale, 30, 18, 18, box)
    o.voxelize_mask(box, mask)
    assert mask.sum() > 50
    assert np.array_equal(g.solid, o.solid)
    assert np.array_equal(g.near, o.near)
    s = o.body_stats()
    assert (g.frontalArea, g.planformArea, g.solidCells, g.rideHeight) == (
        s.frontal_area, s.planform_area, s.solid_cells, s.ride_height)
    assert_bit_exact(g, o, np.float32)


def test_revoxelize_moves_body(both):
    """A second voxelize clears the first body and re-seeds its cells (js/lbm.js:197-202)."""
    g, o = make_pair(both, (24, 12, 12), "f32", "exact", sphere=(8.0, 6.0, 6.0, 3.0))
    g.step_forces(5)
    o.step_forces(5)
    from windtunnel_b200.lbm import sphere_box, sphere_inside
    for s in (g, o):
        s.voxelize(sphere_inside(11.0, 6.0, 6.0, 2.5), sphere_box(11.0, 6.0, 6.0, 2.5), True)
    assert_bit_exact(g, o, np.float32)
    assert_force_close(g.step_forces(5), o.step_forces(5))
    assert_bit_exact(g, o, np.float32)


def test_sample_and_is_solid(both):
    g, o = make_pair(both, (24, 12, 12), "f32", "exact", sphere=(8.0, 6.0, 6.0, 3.0))
    g.step_forces(8)
    o.step_forces(8)
    rng = np.random.default_rng(3)
    pts = rng.uniform(-1, 25, size=(64, 3)) * np.array([1, 0.5, 0.5])
    got = g.sample_points(pts)
    want = np.array([o.sample(*p) for p in pts])
    assert np.array_equal(got, want)
    for p in pts[:16]:
        assert g.isSolid(*p) == o.isSolid(*p)


def test_state_round_trip(both):
    LBM, _ = both
    s = LBM(24, 12, 12)
    apply_case(s, sphere=(8.0, 6.0, 6.0, 3.0))
    s.step_forces(3)
    blob = s.get_state()
    f1 = s.step_forces(5)
    pop1 = s.populations("f", "raw")
    s.set_state(blob)
    assert s.steps == 3
    f2 = s.step_forces(5)
    assert np.array_equal(f1, f2)
    assert np.array_equal(pop1, s.populations("f", "raw"))


def test_populations_set_get_round_trip(both):
    LBM, _ = both
    for storage in ("f32", "f16dev", "f64"):
        s = LBM(12, 8, 8, storage=storage)
        rng = np.random.default_rng(1)
        data = (rng.standard_normal((19, s.n)) * 1e-3).astype(np.float64)
        s.set_populations(data, "g")
        back = s.populations("g", "f64")
        # one rounding to the storage type: half an ulp, relative
        rtol = {"f32": 2.0 ** -24, "f16dev": 2.0 ** -11, "f64": 0.0}[storage]
        assert np.all(np.abs(back - data) <= rtol * np.abs(data))


def test_errors_are_reported(both):
    from windtunnel_b200 import WTError
    from windtunnel_b200 import _lib as W
    LBM, _ = both
    s = LBM(16, 8, 8)
    with pytest.raises(WTError) as e:
        s.tau = 0.4
    assert e.value.code == W.WT_ERR_ARG
    assert s.tau == 0.5035
    with pytest.raises(WTError) as e:
        s.voxelize_mask({"x0": 2, "y0": 2, "z0": 2, "x1": 5, "y1": 5, "z1": 5},
                        np.ones(3, np.uint8))
    assert e.value.code == W.WT_ERR_ARG
    h = LBM(16, 8, 8, storage="f16dev")
    with pytest.raises(WTError) as e:
        h.set_params(math="exact")
    assert e.value.code == W.WT_ERR_UNSUPPORTED
    with pytest.raises(WTError):
        s.set_state(b"\0" * 10)


def test_divergence_is_detected(both):
    """A state with a negative density makes wt_step return WT_ERR_DIVERGED."""
    from windtunnel_b200 import WTError
    from windtunnel_b200 import _lib as W
    LBM, _ = both
    s = LBM(16, 8, 8)
    bad = np.full((19, s.n), -0.2, np.float32)   # rho = 1 + 19*(-0.2) < 0
    s.set_populations(bad, "f")
    with pytest.raises(WTError) as e:
        s.step()
    assert e.value.code == W.WT_ERR_DIVERGED
    s.reset()
    s.step()   # the handle stays usable


def test_reset_matches_oracle(both):
    LBM, OracleLBM = both
    g, o = LBM(20, 10, 10, math="exact"), OracleLBM(20, 10, 10)
    for s in (g, o):
        apply_case(s, sphere=(7.0, 5.0, 5.0, 2.5), amp=0)
        s.step_forces(4)
        s.reset()
    assert_bit_exact(g, o, np.float32)
