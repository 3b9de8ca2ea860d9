"""Host arithmetic of bench.py's long-window accuracy study, on a fake lattice.

The study steps each storage form in chunks and sums the pair-averaged force
(js/main.js:113-127) into blocks; the blocks, their mean and the batch-means
standard error must equal the same statistics computed on the whole series at
once, whatever the chunk boundaries.
"""
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


class FakeLattice:
    """Force series with a drift, a period and noise; step_forces continues it."""
    frontalArea = 120.0

    def __init__(self, offset):
        self.t = 0
        self.offset = offset
        self.rng = np.random.default_rng(7)
        self.series = []

    def set_params(self, **_):
        pass

    def init_eq_noise(self, seed, amp):
        self.noise = (seed, amp)

    def step_forces(self, n):
        t = np.arange(self.t, self.t + n, dtype=np.float64)
        F = np.zeros((n, 3))
        F[:, 0] = self.offset + 1e-3 * np.sin(t / 37.0) + 1e-4 * self.rng.standard_normal(n)
        F[:, 1] = 2e-4 * np.cos(t / 11.0) + (t % 2) * 1e-5   # a parity wobble
        self.t += n
        self.series.append(F)
        return F

    def close(self):
        pass


def test_long_window_blocks_match_the_whole_series(monkeypatch):
    made = {}

    def fake_setup(wl, storage, mm="fast", kernel="auto"):
        lat = FakeLattice(0.2 if storage == "f64" else 0.201)
        made.setdefault(storage, lat)
        return lat

    monkeypatch.setattr(bench, "setup_gpu", fake_setup)
    wl = dict(bench.WORKLOADS["channel256"])
    steps, spinup, block = 25_000, 300, 1000
    out = bench.long_window_accuracy(wl, steps, spinup=spinup, block=block, forms=["f64", "f32"])
    q = 0.5 * wl["u0"] ** 2 * FakeLattice.frontalArea
    for name, storage in (("f64", "f64"), ("f32", "f32")):
        F = np.vstack(made[storage].series)
        assert len(F) == spinup + steps
        pa = 0.5 * (F[1:] + F[:-1])[spinup - 1:]          # the pairs inside the window
        assert len(pa) == steps
        blocks = pa[:, :2].reshape(-1, block, 2).mean(axis=1) / q
        e = out[name]
        assert math.isclose(e["cd"], blocks[:, 0].mean(), rel_tol=1e-12)
        assert math.isclose(e["cl"], blocks[:, 1].mean(), rel_tol=1e-9, abs_tol=1e-15)
        sem = np.std(blocks[:, 0], ddof=1) / math.sqrt(len(blocks))
        assert math.isclose(e["cd_sem"], sem, rel_tol=1e-9)
        b5 = blocks[:, 0].reshape(-1, 5).mean(axis=1)
        assert math.isclose(e["cd_sem_by_block"][str(5 * block)],
                            np.std(b5, ddof=1) / math.sqrt(len(b5)), rel_tol=1e-9)
        assert e["cd_sem_by_block"][str(10 * block)] is not None
    r, f = out["f64"], out["f32"]
    assert math.isclose(f["dcd_rel_vs_f64"], (f["cd"] - r["cd"]) / r["cd"], rel_tol=1e-12)
    assert math.isclose(f["dcd_rel_vs_f64_sem"],
                        math.hypot(f["cd_sem"], r["cd_sem"]) / r["cd"], rel_tol=1e-12)


def test_long_window_noise_seed_keeps_the_body(monkeypatch):
    """--seed re-seeds the initial velocity noise of the workload's lattice
    (its body built from the workload's own seed) and is recorded."""
    made = []

    def fake_setup(wl, storage, mm="fast", kernel="auto"):
        assert wl["seed"] == bench.WORKLOADS["channel256"]["seed"]
        made.append(FakeLattice(0.2))
        return made[-1]

    monkeypatch.setattr(bench, "setup_gpu", fake_setup)
    wl = bench.WORKLOADS["channel256"]
    out = bench.long_window_accuracy(wl, 4000, spinup=10, block=1000, forms=["f32"],
                                     noise_seed=4321)
    assert out["seed"] == 4321
    assert made[0].noise == (4321, wl["amp"])
