"""Partial bounce-back and the discrete adjoint on the GPU, against the oracle.

Bars:
  * the exact-arithmetic partial-bounce-back step (float32 and float64
    storage) is bit-identical to the oracle's (populations, fields); the
    force series agrees to 1e-12 relative (summation order);
  * a field of zeros leaves the step bit-identical to the plain step;
  * the float64 adjoint reproduces the oracle's float64 adjoint (J to 1e-12,
    dJ/ds to 1e-10 relative to the largest component: the force sum's order
    differs) and is independent of the checkpoint interval (bit-identical);
  * the float32 adjoint of the float32 step agrees with the float64 oracle
    gradient to 1e-3 in relative L2;
  * the half-storage adjoint agrees with the oracle's float32-storage
    adjoint to 5e-2 in relative L2 (cosine >= 0.998);
  * the float64 GPU gradient matches central differences of the float64 GPU
    forward (eps 1e-4) to 1e-5 relative.
"""
import numpy as np
import pytest

from lbm_cases import apply_case
from test_adjoint_oracle import smoothed_sphere

pytestmark = pytest.mark.gpu

DIMS = (24, 12, 12)
BOX = (6, 2, 2, 14, 10, 10)
S0 = smoothed_sphere(BOX, (10.0, 6.0, 6.0), 3.0, 1.0, 0.05, seed=7)
CASE = dict(u0=0.05, tau=0.53, side_bc="freeslip")


def _gpu(storage="f32", math="exact", s=S0, **kw):
    from windtunnel_b200 import LBM
    case = dict(CASE, **kw)
    g = LBM(*DIMS, storage=storage, math=math, side_bc=case["side_bc"])
    apply_case(g, **case)
    if s is not None:
        g.set_solid_fraction(BOX, s)
    return g


def _oracle(storage="f32", s=S0, **kw):
    from oracle.oracle import OracleLBM
    case = dict(CASE, **kw)
    o = OracleLBM(*DIMS, storage, side_bc=case["side_bc"])
    apply_case(o, **case)
    if s is not None:
        o.set_solid_fraction(BOX, s)
    return o


@pytest.mark.parametrize("storage", ["f32", "f64"])
@pytest.mark.parametrize("extra", [{}, {"sphere": (19.0, 6.0, 6.0, 2.0)}, {"ground": True}])
def test_pbb_step_bit_identical(wt_lib, oracle_lib, storage, extra):
    g, o = _gpu(storage, **extra), _oracle(storage, **extra)
    fg, fo = g.step_forces(15), o.step_forces(15)
    assert np.abs(fg - fo).max() <= 1e-12 * np.abs(fo).max()
    a, b = g.populations("f", "raw"), o.populations("f", "raw")
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    for x, y in zip(g.fields(), o.fields()):
        assert np.array_equal(x, y)


def test_zero_field_is_the_plain_step(wt_lib):
    g0 = _gpu("f32", s=None)
    g1 = _gpu("f32", s=np.zeros_like(S0))
    assert np.array_equal(g0.step_forces(10), g1.step_forces(10))
    assert np.array_equal(g0.populations("f", "raw"), g1.populations("f", "raw"))


def test_adjoint_f64_reproduces_oracle(wt_lib, oracle_lib):
    N, W = 40, 15
    Jg, gg, st = _gpu("f64").adjoint(N, W, checkpoint=6)
    Jo, go = _oracle("f64").adjoint(N, W)
    assert Jg == pytest.approx(Jo, rel=1e-12)
    assert np.abs(gg - go).max() <= 1e-10 * np.abs(go).max()
    assert st["checkpoints"] == 7 and st["segment"] == 6
    for c in (1, 40, 0):
        _, gc, _ = _gpu("f64").adjoint(N, W, checkpoint=c)
        assert np.array_equal(gc, gg), c


@pytest.mark.parametrize("checkpoint", [6, 40])
def test_adjoint_leaves_the_stepped_state(wt_lib, checkpoint):
    """The lattice ends where step(nsteps) leaves it, whether the last
    interval's states went through the segment store or not."""
    N, W = 40, 15
    g, r = _gpu("f32"), _gpu("f32")
    J, _, _ = g.adjoint(N, W, checkpoint=checkpoint)
    F = r.step_forces(N)
    assert J == pytest.approx(F[-W:, 0].mean(), rel=1e-12)
    assert np.array_equal(g.populations("f", "raw"), r.populations("f", "raw"))
    for x, y in zip(g.fields(), r.fields()):
        assert np.array_equal(x, y)


def test_adjoint_keep_reuses_memory(wt_lib):
    """keep leaves the run's device memory in the lattice: a second and a
    smaller run reuse it and give bit-identical gradients; a larger run
    replaces it; a run without keep frees it."""
    import torch
    N, W = 40, 15
    _, g_ref, st_ref = _gpu("f32").adjoint(N, W, checkpoint=6)
    sim = _gpu("f32")
    start = sim.get_state()
    free0 = torch.cuda.mem_get_info()[0]
    for c, keep in ((6, True), (6, True), (10, True), (3, True), (6, False)):
        sim.set_state(start)
        _, g, st = sim.adjoint(N, W, checkpoint=c, keep=keep)
        if c == 6:
            assert np.array_equal(g, g_ref)
            assert st["device_bytes"] == st_ref["device_bytes"]
    assert torch.cuda.mem_get_info()[0] >= free0 - (8 << 20)


def test_adjoint_f32_close_to_f64(wt_lib, oracle_lib):
    N, W = 40, 15
    _, gf, _ = _gpu("f32", math="fast").adjoint(N, W)
    _, go = _oracle("f64").adjoint(N, W)
    rel_l2 = np.linalg.norm(gf - go) / np.linalg.norm(go)
    assert rel_l2 <= 1e-3, rel_l2


def test_adjoint_f16_close_to_f32(wt_lib, oracle_lib):
    """The half-storage adjoint (half states, float32 adjoint arithmetic; the
    form of the 384x160x160 differentiation workload) against the oracle's
    float32-storage adjoint: the two linearise around trajectories that
    differ by the half rounding of every stored population."""
    N, W = 40, 15
    Jh, gh, st = _gpu("f16dev", math="fast").adjoint(N, W, checkpoint=6)
    Jo, go = _oracle("f32").adjoint(N, W)
    rel_l2 = np.linalg.norm(gh - go) / np.linalg.norm(go)
    cos = float((gh * go).sum() / (np.linalg.norm(gh) * np.linalg.norm(go)))
    assert abs(Jh - Jo) <= 1e-3 * abs(Jo), (Jh, Jo)
    assert rel_l2 <= 5e-2 and cos >= 0.998, (rel_l2, cos)
    assert st["checkpoints"] == 7


def test_adjoint_matches_gpu_central_differences(wt_lib):
    N, W = 40, 15
    _, g, _ = _gpu("f64").adjoint(N, W)
    rng = np.random.default_rng(3)
    eps = 1e-4
    for _ in range(4):
        idx = tuple(int(rng.integers(0, n)) for n in S0.shape)
        sp, sm = S0.copy(), S0.copy()
        sp[idx] += eps
        sm[idx] -= eps
        jp = _gpu("f64", s=sp).step_forces(N)[-W:, 0].mean()
        jm = _gpu("f64", s=sm).step_forces(N)[-W:, 0].mean()
        fd = (jp - jm) / (2 * eps)
        assert abs(g[idx] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(g).max()), (idx, g[idx], fd)


def test_adjoint_errors(wt_lib):
    from windtunnel_b200 import WTError
    from windtunnel_b200 import _lib as W
    g = _gpu("f32", s=None)
    with pytest.raises(WTError) as e:
        g._sbox = BOX
        g.adjoint(10, 5)
    assert e.value.code == W.WT_ERR_STATE
    g.set_solid_fraction(BOX, S0)
    with pytest.raises(WTError):
        g.adjoint(10, 11)
    with pytest.raises(WTError):
        g.set_solid_fraction(BOX, S0 + 2.0)


def test_autograd_function_returns_the_adjoint(wt_lib):
    import torch

    from windtunnel_b200.autograd import drag
    N, W = 30, 10
    g = _gpu("f64", s=None)
    s = torch.tensor(S0, dtype=torch.float64, requires_grad=True)
    J = drag(s, g, BOX, N, W)
    J.backward()
    Jr, gr, _ = _gpu("f64").adjoint(N, W)
    assert float(J) == pytest.approx(Jr, rel=1e-12)
    assert np.array_equal(s.grad.numpy(), gr)
    assert g.steps == N
