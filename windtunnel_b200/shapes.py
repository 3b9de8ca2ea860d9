"""The analytic test bodies of the reference, on the host (js/shapes.js).

The solver's `voxelize(inside, box, ...)` takes a point test; for the
built-in bodies the reference builds it from a list of analytic primitives
(js/shapes.js:16-159) placed by `Body` (js/shapes.js:284-487). This module
restates those closures so the host can evaluate them over a voxelize scan
range (the LBM.voxelize path of this package), with the reference's float64
operation order. The catalogue's numbers are the reference's (its table of
bodies is data the tests and the validation suite run on); the lattice step
itself never runs here.
"""
from __future__ import annotations

import math
from typing import Callable

import numpy as np

PI = math.pi


# ---- NACA 4-digit aerofoil (js/shapes.js:16-26) -----------------------------
def _naca_thickness(xc, t):
    return 5 * t * (0.2969 * np.sqrt(xc) - 0.1260 * xc - 0.3516 * xc * xc +
                    0.2843 * xc * xc * xc - 0.1036 * xc * xc * xc * xc)


def _naca_camber(xc, m, p):
    if m == 0:
        return np.zeros_like(xc)
    return np.where(xc < p, (m / (p * p)) * (2 * p * xc - xc * xc),
                    (m / ((1 - p) * (1 - p))) * ((1 - 2 * p) + 2 * p * xc - xc * xc))


def euler_mat(rx: float, ry: float, rz: float) -> list[float]:
    """3x3 rotation from Euler XYZ, row-major (js/shapes.js:29-39)."""
    a, b = math.cos(rx), math.sin(rx)
    c, d = math.cos(ry), math.sin(ry)
    e, f = math.cos(rz), math.sin(rz)
    ae, af, be, bf = a * e, a * f, b * e, b * f
    return [c * e, -c * f, d,
            af + be * d, ae - bf * d, -b * c,
            bf - ae * d, be + af * d, a * c]


def inside_prim(p: dict, q0, q1, q2):
    """Primitive point test in primitive space (js/shapes.js:42-72), vectorised."""
    s = p["s"]
    t = p["t"]
    if t == "box":
        return (np.abs(q0) <= s[0]) & (np.abs(q1) <= s[1]) & (np.abs(q2) <= s[2])
    if t == "ell":
        a, b, c = q0 / s[0], q1 / s[1], q2 / s[2]
        return a * a + b * b + c * c <= 1
    if t == "cyl":
        return (np.abs(q1) <= s[1]) & ((q0 * q0 + q2 * q2) <= s[0] * s[0])
    if t == "cone":
        r = s[0] * (s[1] - q1) / (2 * s[1])
        return (np.abs(q1) <= s[1]) & ((q0 * q0 + q2 * q2) <= r * r)
    if t == "foil":
        ch, span = s[0], s[2]
        naca = p.get("naca")
        th = naca[2] if naca else 0.12
        m = naca[0] if naca else 0
        pp = naca[1] if naca else 0.4
        xc = (q0 + ch * 0.5) / ch
        ok = (np.abs(q2) <= span * 0.5) & (xc >= 0) & (xc <= 1)
        xs = np.where(ok, xc, 0.0)
        yt = _naca_thickness(xs, th) * ch
        yc = _naca_camber(xs, m, pp) * ch
        return ok & (np.abs(q1 - yc) <= yt)
    return np.zeros_like(q0, dtype=bool)


_HP = PI / 2
# The reference's body catalogue (js/shapes.js:77-159).
BODIES = {
    "sedan": dict(name="Sedan", ground=True, parts=[
        dict(t="ell", c=[0.00, 0.155, 0], s=[0.500, 0.090, 0.185]),
        dict(t="ell", c=[0.05, 0.235, 0], s=[0.250, 0.080, 0.160]),
        dict(t="box", c=[0.00, 0.120, 0], s=[0.430, 0.055, 0.180]),
        dict(t="cyl", wheel=True, c=[-0.290, 0.075, 0.175], s=[0.075, 0.035], r=[_HP, 0, 0]),
        dict(t="cyl", wheel=True, c=[-0.290, 0.075, -0.175], s=[0.075, 0.035], r=[_HP, 0, 0]),
        dict(t="cyl", wheel=True, c=[0.280, 0.075, 0.175], s=[0.075, 0.035], r=[_HP, 0, 0]),
        dict(t="cyl", wheel=True, c=[0.280, 0.075, -0.175], s=[0.075, 0.035], r=[_HP, 0, 0])]),
    "sports": dict(name="Sports car", ground=True, parts=[
        dict(t="ell", c=[0.00, 0.115, 0], s=[0.500, 0.070, 0.200]),
        dict(t="ell", c=[0.07, 0.180, 0], s=[0.190, 0.055, 0.150]),
        dict(t="box", c=[0.00, 0.100, 0], s=[0.450, 0.045, 0.195]),
        dict(t="box", c=[0.450, 0.245, 0], s=[0.045, 0.009, 0.170]),
        dict(t="box", c=[0.430, 0.205, 0.165], s=[0.020, 0.045, 0.008]),
        dict(t="box", c=[0.430, 0.205, -0.165], s=[0.020, 0.045, 0.008]),
        dict(t="cyl", wheel=True, c=[-0.300, 0.070, 0.195], s=[0.070, 0.045], r=[_HP, 0, 0]),
        dict(t="cyl", wheel=True, c=[-0.300, 0.070, -0.195], s=[0.070, 0.045], r=[_HP, 0, 0]),
        dict(t="cyl", wheel=True, c=[0.290, 0.070, 0.195], s=[0.070, 0.050], r=[_HP, 0, 0]),
        dict(t="cyl", wheel=True, c=[0.290, 0.070, -0.195], s=[0.070, 0.050], r=[_HP, 0, 0])]),
    "truck": dict(name="Box truck", ground=True, fill=0.92, parts=[
        dict(t="box", c=[0.100, 0.330, 0], s=[0.380, 0.220, 0.200]),
        dict(t="box", c=[-0.340, 0.190, 0], s=[0.160, 0.110, 0.190]),
        dict(t="cyl", wheel=True, c=[-0.320, 0.080, 0.190], s=[0.080, 0.040], r=[_HP, 0, 0]),
        dict(t="cyl", wheel=True, c=[-0.320, 0.080, -0.190], s=[0.080, 0.040], r=[_HP, 0, 0]),
        dict(t="cyl", wheel=True, c=[0.300, 0.080, 0.190], s=[0.080, 0.040], r=[_HP, 0, 0]),
        dict(t="cyl", wheel=True, c=[0.300, 0.080, -0.190], s=[0.080, 0.040], r=[_HP, 0, 0])]),
    "airplane": dict(name="Airliner", ground=False, ref="planform", fill=0.30, parts=[
        dict(t="ell", c=[0.00, 0, 0], s=[0.500, 0.055, 0.055]),
        dict(t="foil", c=[0.040, -0.020, 0], s=[0.290, 0, 0.900], naca=[0.03, 0.4, 0.15]),
        dict(t="foil", c=[0.430, 0.020, 0], s=[0.130, 0, 0.340], naca=[0.0, 0.4, 0.12]),
        dict(t="foil", c=[0.430, 0.110, 0], s=[0.160, 0, 0.200], naca=[0.0, 0.4, 0.12],
             r=[_HP, 0, 0]),
        dict(t="ell", c=[0.010, -0.058, 0.230], s=[0.090, 0.035, 0.035]),
        dict(t="ell", c=[0.010, -0.058, -0.230], s=[0.090, 0.035, 0.035])]),
    "wing": dict(name="Wing (NACA 4418)", ground=False, ref="planform", fill=0.42, parts=[
        dict(t="foil", c=[0, 0, 0], s=[0.950, 0, 0.900], naca=[0.04, 0.4, 0.18])]),
    "sphere": dict(name="Sphere", ground=False, fill=0.79, parts=[
        dict(t="ell", c=[0, 0, 0], s=[0.28, 0.28, 0.28])]),
    "cube": dict(name="Cube", ground=False, fill=1.0, parts=[
        dict(t="box", c=[0, 0, 0], s=[0.22, 0.22, 0.22])]),
    "cylinder": dict(name="Cylinder (spanwise)", ground=False, fill=1.0, parts=[
        dict(t="cyl", c=[0, 0, 0], s=[0.25, 0.45], r=[_HP, 0, 0])]),
    "teardrop": dict(name="Teardrop", ground=False, fill=0.79, parts=[
        dict(t="ell", c=[-0.220, 0, 0], s=[0.280, 0.130, 0.130]),
        dict(t="cone", c=[0.130, 0, 0], s=[0.130, 0.350], r=[0, 0, -_HP])]),
}


class Body:
    """A positioned, oriented, scaled analytic body (js/shapes.js:284-487)."""

    def __init__(self, key: str):
        self.pos = [0.0, 0.0, 0.0]
        self.scale = 30.0
        self.pitch = 0.0
        self.yaw = 0.0
        self.set_type(key)

    def set_type(self, key: str) -> None:
        self.key = key
        self.defn = BODIES[key]
        self.parts = []
        for p in self.defn["parts"]:
            q = dict(p)
            q["r"] = p.get("r", [0, 0, 0])
            q["m"] = euler_mat(*q["r"])
            self.parts.append(q)
        e = [0.0, 0.0, 0.0]
        for p in self.parts:
            s = p["s"]
            if p["t"] in ("box", "ell"):
                h = [s[0], s[1], s[2]]
            elif p["t"] in ("cyl", "cone"):
                h = [s[0], s[1], s[0]]
            elif p["t"] == "foil":
                h = [s[0] * 0.5, s[0] * 0.22, s[2] * 0.5]
            else:
                h = [0, 0, 0]
            m = p["m"]
            for i in range(3):
                w = abs(m[i * 3]) * h[0] + abs(m[i * 3 + 1]) * h[1] + abs(m[i * 3 + 2]) * h[2]
                e[i] = max(e[i], abs(p["c"][i]) + w)
        self.ext = e
        self.radius = max(e)

    @property
    def ground(self) -> bool:
        return bool(self.defn["ground"])

    @property
    def ref(self) -> str:
        return self.defn.get("ref", "frontal")

    def fit(self, nx: int, ny: int, nz: int) -> float:
        """Size by frontal blockage and clearances (js/shapes.js:338-350)."""
        e = self.ext
        hy = e[1] if self.ground else 2 * e[1]
        wz = 2 * e[2]
        fill = self.defn.get("fill") or 0.7
        blockage = math.sqrt(0.10 * ny * nz / (hy * wz * fill))
        self.scale = min(blockage, nx * 0.34 / (2 * e[0]), ny * 0.55 / hy, nz * 0.75 / wz)
        return self.scale

    @property
    def M(self) -> list[float]:
        """Body -> world rotation, yaw about y then pitch about z (js/shapes.js:353-362)."""
        cy, sy = math.cos(self.yaw), math.sin(self.yaw)
        cp, sp = math.cos(self.pitch), math.sin(self.pitch)
        return [cy * cp, -cy * sp, sy, sp, cp, 0, -sy * cp, sy * sp, cy]

    def make_test(self) -> Callable:
        """inside(X, Y, Z) in lattice coordinates (js/shapes.js:391-408), vectorised."""
        M, P, inv = self.M, list(self.pos), 1 / self.scale
        parts = self.parts

        def inside(X, Y, Z):
            X, Y, Z = (np.asarray(v, np.float64) for v in (X, Y, Z))
            dx, dy, dz = X - P[0], Y - P[1], Z - P[2]
            l0 = (M[0] * dx + M[3] * dy + M[6] * dz) * inv
            l1 = (M[1] * dx + M[4] * dy + M[7] * dz) * inv
            l2 = (M[2] * dx + M[5] * dy + M[8] * dz) * inv
            hit = np.zeros(np.shape(l0), dtype=bool)
            for p in parts:
                m, c = p["m"], p["c"]
                ax, ay, az = l0 - c[0], l1 - c[1], l2 - c[2]
                q0 = m[0] * ax + m[3] * ay + m[6] * az
                q1 = m[1] * ax + m[4] * ay + m[7] * az
                q2 = m[2] * ax + m[5] * ay + m[8] * az
                hit |= inside_prim(p, q0, q1, q2)
            return hit
        return inside

    def box(self) -> dict:
        """Tight AABB in lattice coordinates plus 2 cells (js/shapes.js:473-486)."""
        M, e, s, P = self.M, self.ext, self.scale, self.pos
        w = [s * (abs(M[i * 3]) * e[0] + abs(M[i * 3 + 1]) * e[1] + abs(M[i * 3 + 2]) * e[2]) + 2
             for i in range(3)]
        return {"x0": P[0] - w[0], "x1": P[0] + w[0], "y0": P[1] - w[1], "y1": P[1] + w[1],
                "z0": P[2] - w[2], "z1": P[2] + w[2]}
