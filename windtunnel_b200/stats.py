"""Force statistics of a run: the reference's measurement pipeline on the host.

Restates js/main.js:59-212: the settle window, the running EMA, pair
averaging of consecutive steps (which cancels the lattice's odd/even force
oscillation, js/main.js:95-104), the ring of post-settle coefficient samples
(stored as float32, js/main.js:65-66), the 16-block blocking estimate of the
standard error (js/main.js:163-191) and the drift / convergence verdict
(js/main.js:193-212). `ForceStats.accumulate` is fed one step's force at a
time, exactly like the reference's per-step `accumulate()`; `series_stats`
applies the same pipeline to a whole force series (e.g. `LBM.step_forces`).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

HIST = 6000          # js/main.js:65
CAP_MAX = 250000     # js/main.js:74
SETTLE_DEFAULT = 150  # js/main.js:83


@dataclass
class Block:
    mean: float
    sem: float
    blocked: bool
    used: int | None = None


def block_stats(x, n: int | None = None) -> Block:
    """Mean and blocking-method standard error, js/main.js:163-191."""
    x = np.asarray(x, np.float64)
    n = len(x) if n is None else n
    B = 16
    bl = n // B
    if bl < 4:
        m = 0.0
        for i in range(n):
            m += x[i]
        m /= n
        v = 0.0
        for i in range(n):
            d = x[i] - m
            v += d * d
        return Block(m, math.sqrt(v / max(1, n - 1) / n), False)
    used = B * bl
    bm = np.zeros(B)
    mean = 0.0
    for b in range(B):
        s = 0.0
        for i in range(b * bl, (b + 1) * bl):
            s += x[i]
        bm[b] = s / bl
        mean += bm[b]
    mean /= B
    v = 0.0
    for b in range(B):
        d = bm[b] - mean
        v += d * d
    return Block(mean, math.sqrt(v / (B - 1) / B), True, used)


@dataclass
class RunStats:
    n: int
    cd: Block
    cl: Block
    cy: Block
    drift: float
    rel: float
    state: str


@dataclass
class ForceStats:
    """The reference's live statistics state (js/main.js:59-212)."""
    u0: float
    ref_area: float                      # frontalArea or planformArea, in cells
    settle: int = SETTLE_DEFAULT
    force_ema: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    f_count: int = 0
    h_n: int = 0
    have_prev: bool = False
    prev: list = field(default_factory=lambda: [0.0, 0.0, 0.0])

    def __post_init__(self):
        self.h_cd = np.zeros(HIST, np.float32)
        self.h_cl = np.zeros(HIST, np.float32)
        self.h_cy = np.zeros(HIST, np.float32)
        self.capture = None

    def reset(self, settle: int | None = None) -> None:
        """resetAverages(), js/main.js:78-84."""
        self.force_ema = [0.0, 0.0, 0.0]
        self.f_count = 0
        self.h_n = 0
        self.have_prev = False
        self.settle = SETTLE_DEFAULT if settle is None else settle

    def start_capture(self) -> None:
        self.capture = {"cd": [], "cl": [], "cy": []}

    def accumulate(self, force) -> None:
        """Fold one step's force in, js/main.js:106-111."""
        if self.settle > 0:
            self.settle -= 1
            return
        self.f_count += 1
        a = 1 / min(self.f_count, 500)
        for k in range(3):
            self.force_ema[k] += (force[k] - self.force_ema[k]) * a
        self._push(force)

    def _push(self, force) -> None:
        """pushSample(), js/main.js:113-127 (pair-averaged coefficients)."""
        if not self.have_prev:
            self.prev = [float(force[0]), float(force[1]), float(force[2])]
            self.have_prev = True
            return
        q = 0.5 * self.u0 * self.u0 * self.ref_area
        i = self.h_n % HIST
        cd = 0.5 * (force[0] + self.prev[0]) / q
        cl = 0.5 * (force[1] + self.prev[1]) / q
        cy = 0.5 * (force[2] + self.prev[2]) / q
        self.h_cd[i] = cd
        self.h_cl[i] = cl
        self.h_cy[i] = cy
        self.prev = [float(force[0]), float(force[1]), float(force[2])]
        self.h_n += 1
        if self.capture is not None and len(self.capture["cd"]) < CAP_MAX:
            self.capture["cd"].append(cd)
            self.capture["cl"].append(cl)
            self.capture["cy"].append(cy)

    def ordered(self, src: np.ndarray) -> np.ndarray:
        """The ring in chronological order, js/main.js:155-161."""
        n = min(self.h_n, HIST)
        s = 0 if self.h_n <= HIST else self.h_n % HIST
        return np.array([src[(s + i) % HIST] for i in range(n)], np.float64)

    def run_stats(self) -> RunStats | None:
        """runStats(), js/main.js:193-212."""
        x = self.ordered(self.h_cd)
        n = len(x)
        if n < 60:
            return None
        cd = block_stats(x, n)
        h = n >> 1
        m1 = sum(x[i] for i in range(h)) / h
        m2 = sum(x[i] for i in range(h, n)) / (n - h)
        drift = abs(m1 - m2)
        cl = block_stats(self.ordered(self.h_cl))
        cy = block_stats(self.ordered(self.h_cy))
        rel = 1.96 * cd.sem / max(1e-9, abs(cd.mean))
        drifting = drift > 2.5 * cd.sem
        state = ("averaging" if n < 400 else "drifting" if drifting else
                 "converged" if rel < 0.03 else "noisy")
        return RunStats(n, cd, cl, cy, drift, rel, state)


def series_stats(forces, u0: float, ref_area: float, settle: int = SETTLE_DEFAULT) -> RunStats | None:
    """Run a whole (steps, 3) force series through the live pipeline."""
    st = ForceStats(u0=u0, ref_area=ref_area, settle=settle)
    for f in np.asarray(forces, np.float64):
        st.accumulate(f)
    return st.run_stats()


def window_coefficients(forces, u0: float, ref_area: float, window: int) -> dict:
    """Pair-averaged Cd / Cl / Cy over the last `window` samples, with blocking SEMs.

    This is the capture statistic the benchmark reports: the same pair
    averaging as js/main.js:113-127 over an explicit window, without the
    float32 ring (the values stay float64).
    """
    f = np.asarray(forces, np.float64)
    q = 0.5 * u0 * u0 * ref_area
    pa = 0.5 * (f[1:] + f[:-1]) / q
    w = pa[-window:]
    out = {}
    for k, name in enumerate(("cd", "cl", "cy")):
        b = block_stats(w[:, k])
        out[name] = b.mean
        out[name + "_sem"] = b.sem
    return out
