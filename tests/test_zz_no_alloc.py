"""wt_step_noalloc: the step that allocates nothing, against wt_step.

Some hosts cannot let the library call cudaMalloc while they run: one whose
own memory pool already holds the device's memory, or a frame loop that must
not stall on an allocation. wt_step_noalloc serves them with a fixed device
array. Here two lattices get the same set-up; one advances with wt_step, the
other with wt_step_noalloc, both called straight through the C ABI, twice in
a row. The force series and the populations must agree (the two calls run
the same kernels in the same order, so they agree exactly; the tolerance
below is the fast-collision test tolerance), and the free device memory must
not move across a wt_step_noalloc call. The file is named to be collected
last, so that it also runs after every other test has used the device.
"""
import ctypes as C

import numpy as np
import pytest

from lbm_cases import CFG0, apply_case, rel_linf, spinning_sphere_wallvel

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _lattice(storage, ground=False, math=None, moving=False):
    from windtunnel_b200.lbm import LBM
    sim = LBM(CFG0["nx"], CFG0["ny"], CFG0["nz"], storage=storage)
    cx, cy, cz, r = CFG0["sphere"]
    apply_case(sim, u0=CFG0["u0"], tau=CFG0["tau"], csm=CFG0["csm"], lam=CFG0["lam"],
               sphere=CFG0["sphere"], ground=ground or moving, seed=CFG0["seed"],
               amp=CFG0["amp"], math=math, roadVel=0.03 if moving else 0.0,
               wallVel=spinning_sphere_wallvel(cx, cy, cz, 0.01) if moving else None)
    return sim


def _steps(fn, sim, n):
    out = np.empty(3 * n, np.float64)
    code = fn(sim._h, n, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert code == 0, _err(sim)
    return out.reshape(n, 3)


def _err(sim):
    from windtunnel_b200 import _lib
    return _lib.lib().wt_last_error(sim._h).decode()


@pytest.mark.parametrize("storage,ground,math,moving", [
    ("f32", False, None, False), ("f32", True, None, False), ("f32", False, "exact", False),
    ("f32", False, None, True), ("f16dev", False, None, False), ("f64", False, None, False)])
def test_noalloc_matches_step_two_calls(wt_lib, storage, ground, math, moving):
    import torch
    a = _lattice(storage, ground, math, moving)
    b = _lattice(storage, ground, math, moving)
    assert bool(b.movingWalls) == moving
    assert wt_lib.wt_step_noalloc(b._h, 0, None) == 0, _err(b)   # set-up call
    for n in (37, 20):              # two calls in a row, neither a multiple of the chunk
        fa = _steps(wt_lib.wt_step, a, n)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        fb = _steps(wt_lib.wt_step_noalloc, b, n)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0   # nothing allocated inside the call
        assert np.abs(fa).max() > 0
        assert rel_linf(fb, fa) <= TOL
        assert rel_linf(b.populations("f"), a.populations("f")) <= TOL
        assert b.steps == a.steps and b.parity == a.parity
        assert b.force == pytest.approx(a.force, rel=TOL)
    assert rel_linf(b.ux, a.ux) <= TOL


def test_noalloc_rejects_sizes_beyond_its_scratch(wt_lib):
    from windtunnel_b200 import _lib
    sim = _lattice("f32")
    assert wt_lib.wt_step_noalloc(sim._h, 4097, None) == _lib.WT_ERR_ARG
    assert "0..4096" in _err(sim)
    assert wt_lib.wt_step_noalloc(sim._h, -1, None) == _lib.WT_ERR_ARG
    assert sim.steps == 0
    assert wt_lib.wt_step_noalloc(sim._h, 0, None) == _lib.WT_OK
    s = np.full((4, 4, 4), 0.5)
    sim.set_solid_fraction((60, 30, 30, 64, 34, 34), s)
    assert wt_lib.wt_step_noalloc(sim._h, 1, None) == _lib.WT_ERR_UNSUPPORTED
    assert "partial bounce-back" in _err(sim)
    assert sim.steps == 0
