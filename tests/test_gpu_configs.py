"""Parity on the benchmark workloads themselves, against the CPU oracle.

The small-lattice parity tests cover every rule of the step; these run the
lattices the bench measures, built the way the bench builds them (the
20000-triangle hull through Voxel.build and the device lookup on the GPU,
the oracle's Voxel.build and lookup on the CPU):

  * 256x128x128 hull channel (Re 2000, LES, free-slip), 100 steps:
    occupancy, near flags and body statistics bit-exact; the exact form
    (float64 collision, float32 storage) bit-identical in both population
    buffers and the fields, forces to 1e-12; the float32 collision (the
    bench's form) within FAST_TOL on u and rho and 1e-3 on the
    pair-averaged drag; half storage (the AUTO kernel) within HALF_TOL on u
    and 1e-2 on the drag.
  * 512x192x192 hull channel, half storage (the AUTO kernel), 20 steps
    against the float32 oracle: u within HALF_TOL, drag within 1e-2.
"""
import os

import numpy as np
import pytest

from lbm_cases import oracle_channel, pair_average, rel_linf

pytestmark = pytest.mark.gpu

FAST_TOL = 2e-4      # float32 collision vs the reference's float64 arithmetic, u and rho
HALF_TOL = 2e-2      # half-precision deviations vs float32 storage, u
THREADS = max(1, min(16, os.cpu_count() or 1))


@pytest.fixture(scope="module")
def channel256(wt_lib, oracle_lib):
    from windtunnel_b200.workloads import WORKLOADS
    wl = WORKLOADS["channel256"]
    o = oracle_channel(wl)
    occupancy = (o.solid.copy(), o.near.copy(), o.body_stats())
    forces = o.step_forces(100, threads=THREADS)
    out = dict(wl=wl, occupancy=occupancy, forces=forces, fields=o.fields(),
               f=o.populations("f", "raw"), g=o.populations("g", "raw"), steps=o.steps,
               parity=o.parity)
    o.close()
    return out


def _drag(forces, window=50):
    return pair_average(np.asarray(forces)[:, 0])[-window:].mean()


def test_channel256_occupancy_bit_exact(channel256):
    from windtunnel_b200.workloads import channel_lattice
    g = channel_lattice(channel256["wl"], "f32", "exact")
    solid, near, st = channel256["occupancy"]
    assert np.array_equal(g.solid, solid)
    assert np.array_equal(g.near, near)
    assert (g.frontalArea, g.planformArea, g.solidCells, g.rideHeight) == (
        st.frontal_area, st.planform_area, st.solid_cells, st.ride_height)
    assert solid.sum() > 10000


def test_channel256_exact_bit_identical(channel256):
    from windtunnel_b200.workloads import channel_lattice
    g = channel_lattice(channel256["wl"], "f32", "exact")
    fg = g.step_forces(100)
    fo = channel256["forces"]
    assert np.abs(fg - fo).max() <= 1e-12 * np.abs(fo).max()
    assert g.steps == channel256["steps"] and g.parity == channel256["parity"]
    for which in ("f", "g"):
        a = g.populations(which, "raw")
        assert np.array_equal(a.view(np.uint32), channel256[which].view(np.uint32)), which
    for a, b in zip(g.fields(), channel256["fields"]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_channel256_fast_within_tolerance(channel256):
    from windtunnel_b200.workloads import channel_lattice
    g = channel_lattice(channel256["wl"], "f32", "fast")
    fg = g.step_forces(100)
    gu, ou = g.fields(), channel256["fields"]
    for name, a, b in zip(("ux", "uy", "uz"), gu[:3], ou[:3]):
        assert rel_linf(a, b) < FAST_TOL, name
    assert np.abs(gu[3] - ou[3]).max() < FAST_TOL * 0.06
    fo = channel256["forces"]
    assert abs(_drag(fg) - _drag(fo)) <= 1e-3 * abs(_drag(fo))


@pytest.mark.parametrize("kernel", ["auto", "lean"])
def test_channel256_half_within_tolerance(channel256, kernel):
    from windtunnel_b200.workloads import channel_lattice
    g = channel_lattice(channel256["wl"], "f16dev", "fast", kernel=kernel)
    fg = g.step_forces(100)
    gu, ou = g.fields(), channel256["fields"]
    assert rel_linf(gu[0], ou[0]) < HALF_TOL
    fo = channel256["forces"]
    assert abs(_drag(fg) - _drag(fo)) <= 1e-2 * abs(_drag(fo))


def test_channel512_half_within_tolerance(wt_lib, oracle_lib):
    from windtunnel_b200.workloads import WORKLOADS, channel_lattice
    wl = WORKLOADS["channel512"]
    o = oracle_channel(wl)
    fo = o.step_forces(20, threads=THREADS)
    ou = o.fields()
    solid = o.solid
    o.close()
    g = channel_lattice(wl, "f16dev", "fast")
    assert np.array_equal(g.solid, solid)
    fg = g.step_forces(20)
    gu = g.fields()
    assert rel_linf(gu[0], ou[0]) < HALF_TOL
    assert abs(_drag(fg, 10) - _drag(fo, 10)) <= 1e-2 * abs(_drag(fo, 10))
