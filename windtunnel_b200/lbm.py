"""Host mirror of windtunnel's solver interface over libwt.so.

`LBM` keeps the property and method names of the reference class in
js/lbm.js:51-550 (`u0`, `tau`, `les`, `csm`, `trt`, `lambda`, `movingWalls`,
`reset()`, `voxelize()`, `step()`, `force`, `ux/uy/uz/rho`, `solid`, `near`,
`frontalArea`, `planformArea`, `solidCells`, `rideHeight`, `steps`, `nu`,
`sample()`, `isSolid()`, `f`/`g`), and `step_batch(n)` stands for
`LBMPool.Pool.step(n)` (js/pool.js:97-125), returning the per-step force
series. Every call goes through the C ABI; nothing here computes the flow.
Errors raise `WTError`, as the reference throws `Error`s.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Iterable, Sequence

import numpy as np

from . import _lib as W
from ._lib import WTError, check, lib

Q = 19
EX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0], np.int32)
EY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1], np.int32)
EZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1], np.int32)
OPP = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17], np.int32)
WEIGHTS = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float64)

FLUID, SOLID_OBJ, SOLID_WALL = W.WT_FLUID, W.WT_SOLID_OBJ, W.WT_SOLID_WALL

STORAGE = {"f32": W.WT_STORE_F32, "f16dev": W.WT_STORE_F16DEV, "f64": W.WT_STORE_F64}
MATH = {"fast": W.WT_MATH_FAST, "exact": W.WT_MATH_EXACT}
SIDE = {"eq": W.WT_SIDE_EQ, "freeslip": W.WT_SIDE_FREESLIP}
KERNEL = {"auto": W.WT_KERNEL_AUTO, "direct": W.WT_KERNEL_DIRECT, "lean": W.WT_KERNEL_LEAN,
          "pair": W.WT_KERNEL_PAIR}
_STORE_DTYPE = {W.WT_STORE_F32: np.float32, W.WT_STORE_F16DEV: np.float16,
                W.WT_STORE_F64: np.float64}


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _box6(box) -> np.ndarray:
    """A reference box ({x0,y0,z0,x1,y1,z1}, js/shapes.js:473-486) as 6 doubles."""
    if isinstance(box, dict):
        v = [box[k] for k in ("x0", "y0", "z0", "x1", "y1", "z1")]
    elif hasattr(box, "x0"):
        v = [getattr(box, k) for k in ("x0", "y0", "z0", "x1", "y1", "z1")]
    else:
        v = list(box)
    if len(v) != 6:
        raise ValueError("box needs x0, y0, z0, x1, y1, z1")
    return np.ascontiguousarray(v, dtype=np.float64)


class LBM:
    """D3Q19 lattice on the current CUDA device (the reference `new LBM(nx, ny, nz)`)."""

    Q = Q
    EX = EX
    EY = EY
    EZ = EZ
    W = WEIGHTS
    FLUID = FLUID
    SOLID_OBJ = SOLID_OBJ
    SOLID_WALL = SOLID_WALL

    def __init__(self, nx: int, ny: int, nz: int, storage: str = "f32", math: str = "fast",
                 side_bc: str = "eq", kernel: str = "auto"):
        if storage not in STORAGE:
            raise ValueError(f"storage must be one of {sorted(STORAGE)}")
        L = lib()
        h = C.c_void_p()
        check(L.wt_create(int(nx), int(ny), int(nz), STORAGE[storage], C.byref(h)), None)
        self._h = h
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.n = self.nx * self.ny * self.nz
        self.storage = storage
        self._p = W.default_params()
        self._p.math = MATH[math]
        self._p.side_bc = SIDE[side_bc]
        self._p.kernel = KERNEL[kernel]
        self._push()
        self._fields_at = -1
        self._fields = None

    # ---- lifetime --------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().wt_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _call(self, fn, *args) -> int:
        return check(fn(self._h, *args), self._h)

    # ---- parameters (js/lbm.js:95, :106-111) -----------------------------------------
    def _push(self) -> None:
        self._call(lib().wt_set_params, C.byref(self._p))

    def _pull(self) -> None:
        self._call(lib().wt_get_params, C.byref(self._p))

    def _param(name, conv=float):
        def get(self):
            self._pull()
            return conv(getattr(self._p, name))

        def set_(self, v):
            self._pull()
            old = getattr(self._p, name)
            setattr(self._p, name, type(old)(v) if not isinstance(old, float) else float(v))
            try:
                self._push()
            except WTError:
                setattr(self._p, name, old)
                raise
        return property(get, set_)

    u0 = _param("u0")
    tau = _param("tau")
    les = _param("les", bool)
    csm = _param("csm")
    trt = _param("trt", bool)
    lambda_ = _param("lambda_")
    movingWalls = _param("moving_walls", bool)
    side_bc = _param("side_bc", int)
    math = _param("math", int)
    kernel = _param("kernel", int)
    f16_rounding = _param("f16_rounding", int)
    del _param

    @property
    def nu(self) -> float:
        """Kinematic viscosity, js/lbm.js:143."""
        return (self.tau - 0.5) / 3

    def params(self) -> W.wt_params:
        self._pull()
        p = W.wt_params()
        C.pointer(p)[0] = self._p
        return p

    def set_params(self, **kw) -> None:
        """Assign several public fields at once (e.g. u0=0.05, tau=0.512)."""
        self._pull()
        old = W.wt_params()
        C.pointer(old)[0] = self._p
        for k, v in kw.items():
            key = {"lambda": "lambda_", "movingWalls": "moving_walls"}.get(k, k)
            if key == "side_bc" and isinstance(v, str):
                v = SIDE[v]
            if key == "math" and isinstance(v, str):
                v = MATH[v]
            if key == "kernel" and isinstance(v, str):
                v = KERNEL[v]
            if key == "f16_rounding" and isinstance(v, str):
                v = {"nearest": W.WT_ROUND_NEAREST, "stochastic": W.WT_ROUND_STOCHASTIC}[v]
            cur = getattr(self._p, key)
            setattr(self._p, key, float(v) if isinstance(cur, float) else int(v))
        try:
            self._push()
        except WTError:
            C.pointer(self._p)[0] = old
            raise

    # ---- state -----------------------------------------------------------------------
    def reset(self) -> None:
        """js/lbm.js:164-174."""
        self._call(lib().wt_reset)
        self._fields_at = -1

    def init_eq_noise(self, seed: int, amp: float) -> None:
        """reset() plus seeded velocity noise of amplitude amp on fluid cells."""
        self._call(lib().wt_init_eq_noise, C.c_uint64(seed), float(amp))
        self._fields_at = -1

    # ---- occupancy (js/lbm.js:191-266) -------------------------------------------------
    def voxel_range(self, box) -> tuple[int, int, int, int, int, int]:
        rg = (C.c_int * 6)()
        self._call(lib().wt_voxel_range, _dptr(_box6(box)), rg)
        return tuple(rg)

    def voxelize(self, inside, box, ground: bool = False,
                 wallVel: Callable | None = None, roadVel: float = 0.0) -> None:
        """Rasterise a body given by a point test inside(x, y, z) in lattice units.

        `inside` is evaluated at the cell centres of the scan range of `box`
        (js/lbm.js:225-229) on the host, vectorised when it accepts numpy
        arrays; `wallVel(x, y, z, out)` likewise for moving surfaces.
        """
        b = _box6(box)
        x0, x1, y0, y1, z0, z1 = self.voxel_range(b)
        ex, ey, ez = max(0, x1 - x0 + 1), max(0, y1 - y0 + 1), max(0, z1 - z0 + 1)
        zz, yy, xx = np.meshgrid(np.arange(z0, z0 + ez) + 0.5, np.arange(y0, y0 + ey) + 0.5,
                                 np.arange(x0, x0 + ex) + 0.5, indexing="ij")
        X, Y, Z = xx.ravel(), yy.ravel(), zz.ravel()
        mask = _evaluate_inside(inside, X, Y, Z)
        wall_set = wall_vel = None
        if wallVel is not None:
            wall_set = np.zeros(mask.size, np.uint8)
            wall_vel = np.zeros((mask.size, 3), np.float64)
            out = [0.0, 0.0, 0.0]
            for m in np.flatnonzero(mask):
                if wallVel(float(X[m]), float(Y[m]), float(Z[m]), out):
                    wall_set[m] = 1
                    wall_vel[m] = out
        self.voxelize_mask(b, mask, ground, wall_set, wall_vel, roadVel)

    def voxelize_mask(self, box, mask: np.ndarray, ground: bool = False,
                      wall_set: np.ndarray | None = None, wall_vel: np.ndarray | None = None,
                      roadVel: float = 0.0) -> None:
        b = _box6(box)
        m = np.ascontiguousarray(mask, dtype=np.uint8).ravel()
        ws = wv = None
        if wall_set is not None:
            ws = np.ascontiguousarray(wall_set, dtype=np.uint8).ravel()
            wv = np.ascontiguousarray(wall_vel, dtype=np.float64).ravel()
        self._call(lib().wt_voxelize_mask, _dptr(b), m.ctypes.data_as(C.POINTER(C.c_uint8)),
                   m.size,
                   ws.ctypes.data_as(C.POINTER(C.c_uint8)) if ws is not None else None,
                   _dptr(wv) if wv is not None else None, int(bool(ground)), float(roadVel or 0))
        self._fields_at = -1

    def voxelize_grid(self, grid: np.ndarray, gmin: Sequence[float], ginv: float,
                      M: Sequence[float], P: Sequence[float], scale: float, box,
                      ground: bool = False, roadVel: float = 0.0) -> None:
        """voxelize() with the voxel-backed Body.makeTest() closure evaluated on the device.

        grid is the body-space occupancy (gnz, gny, gnx) of js/voxel.js:89-101;
        M, P and scale place it as js/shapes.js:365-388 does.
        """
        g = np.ascontiguousarray(grid, dtype=np.uint8)
        gnz, gny, gnx = g.shape
        self._call(lib().wt_voxelize_grid, g.ctypes.data_as(C.POINTER(C.c_uint8)), gnx, gny, gnz,
                   _dptr(np.ascontiguousarray(gmin, np.float64)), float(ginv),
                   _dptr(np.ascontiguousarray(M, np.float64)),
                   _dptr(np.ascontiguousarray(P, np.float64)), float(scale), _dptr(_box6(box)),
                   int(bool(ground)), float(roadVel or 0))
        self._fields_at = -1

    def _stats(self) -> W.wt_body_stats:
        s = W.wt_body_stats()
        self._call(lib().wt_get_body_stats, C.byref(s))
        return s

    @property
    def frontalArea(self) -> int:
        return self._stats().frontal_area

    @property
    def planformArea(self) -> int:
        return self._stats().planform_area

    @property
    def solidCells(self) -> int:
        return self._stats().solid_cells

    @property
    def rideHeight(self) -> int:
        return self._stats().ride_height

    @property
    def ground(self) -> bool:
        return bool(self._stats().ground)

    # ---- stepping (js/lbm.js:285-291, js/pool.js:97-125) ------------------------------
    def step(self) -> None:
        """Advance one lattice time step; `force` then holds its momentum exchange."""
        self._call(lib().wt_step, 1, None)

    def step_batch(self, n: int) -> list[list[float]]:
        """Advance n steps; returns the per-step force series [[fx,fy,fz], ...]."""
        n = int(n)
        if n <= 0:
            return []
        out = np.empty(3 * n, np.float64)
        self._call(lib().wt_step, n, _dptr(out))
        return out.reshape(n, 3).tolist()

    def step_forces(self, n: int) -> np.ndarray:
        """As step_batch, as an (n, 3) float64 array."""
        out = np.empty(3 * int(n), np.float64)
        if n > 0:
            self._call(lib().wt_step, int(n), _dptr(out))
        return out.reshape(int(n), 3)

    @property
    def force(self) -> np.ndarray:
        out = np.empty(3, np.float64)
        self._call(lib().wt_get_force, _dptr(out))
        return out

    @property
    def steps(self) -> int:
        s = C.c_int64()
        self._call(lib().wt_get_steps, C.byref(s), None)
        return s.value

    @property
    def parity(self) -> int:
        p = C.c_int()
        self._call(lib().wt_get_steps, None, C.byref(p))
        return p.value

    # ---- fields (js/lbm.js:82-88) ------------------------------------------------------
    def fields(self) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        """(ux, uy, uz, rho), each a float32 array of n cells, fresh from the device."""
        a = [np.empty(self.n, np.float32) for _ in range(4)]
        self._call(lib().wt_get_fields, *[x.ctypes.data_as(C.POINTER(C.c_float)) for x in a])
        return tuple(a)

    def _cached_fields(self):
        st = self.steps
        if self._fields is None or self._fields_at != st:
            self._fields = self.fields()
            self._fields_at = st
        return self._fields

    @property
    def ux(self) -> np.ndarray:
        return self._cached_fields()[0]

    @property
    def uy(self) -> np.ndarray:
        return self._cached_fields()[1]

    @property
    def uz(self) -> np.ndarray:
        return self._cached_fields()[2]

    @property
    def rho(self) -> np.ndarray:
        return self._cached_fields()[3]

    @property
    def solid(self) -> np.ndarray:
        out = np.empty(self.n, np.uint8)
        self._call(lib().wt_get_solid, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out

    @property
    def near(self) -> np.ndarray:
        out = np.empty(self.n, np.uint8)
        self._call(lib().wt_get_near, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out

    # ---- populations (js/lbm.js:131-132) -------------------------------------------------
    def populations(self, which: str = "f", dtype: str = "f32") -> np.ndarray:
        """Stored deviations f_q - w_q as a (19, n) array (dtype 'f32', 'f64' or 'raw')."""
        code = {"f32": W.WT_STORE_F32, "f64": W.WT_STORE_F64}.get(dtype)
        if dtype == "raw":
            code = STORAGE[self.storage]
        npd = _STORE_DTYPE[code]
        out = np.empty(19 * self.n, npd)
        self._call(lib().wt_get_populations, W.WT_BUF_F if which == "f" else W.WT_BUF_G, code,
                   out.ctypes.data, out.nbytes)
        return out.reshape(19, self.n)

    def set_populations(self, data: np.ndarray, which: str = "f") -> None:
        a = np.ascontiguousarray(data)
        code = {np.dtype(np.float32): W.WT_STORE_F32, np.dtype(np.float64): W.WT_STORE_F64,
                np.dtype(np.float16): W.WT_STORE_F16DEV}[a.dtype]
        self._call(lib().wt_set_populations, W.WT_BUF_F if which == "f" else W.WT_BUF_G, code,
                   a.ctypes.data, a.nbytes)

    @property
    def f(self) -> np.ndarray:
        return self.populations("f")

    @property
    def g(self) -> np.ndarray:
        return self.populations("g")

    # ---- visualisation arithmetic (js/main.js:691-709, :925-968) ---------------------------
    def slice(self, plane: str = "xy", k: int | None = None, field: str = "speed") -> np.ndarray:
        """The slice view's scalar on plane 'xy' (z = k) or 'xz' (y = k): field 'speed'
        (|u|/u0), 'pressure' (Cp) or 'vorticity' (/u0); NaN on solid cells."""
        p = {"xy": 0, "xz": 1}[plane]
        if k is None:
            k = (self.nz if p == 0 else self.ny) // 2
        h = self.ny if p == 0 else self.nz
        out = np.empty((h, self.nx), np.float32)
        f = {"speed": 0, "pressure": 1, "vorticity": 2}[field]
        self._call(lib().wt_slice, p, int(k), f, out.ctypes.data_as(C.POINTER(C.c_float)),
                   out.size)
        return out

    def advect(self, xyz: np.ndarray, kstep: float):
        """One smoke-particle step: (new positions (n, 3), expired (n,) bool, speed (n,))."""
        p = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3).copy()
        n = p.shape[0]
        expired = np.zeros(n, np.uint8)
        speed = np.zeros(n, np.float32)
        self._call(lib().wt_advect, _dptr(p), n, float(kstep),
                   expired.ctypes.data_as(C.POINTER(C.c_uint8)),
                   speed.ctypes.data_as(C.POINTER(C.c_float)))
        return p, expired.astype(bool), speed

    # ---- partial bounce-back and its adjoint (no reference counterpart) ------------------
    def set_solid_fraction(self, box, s) -> None:
        """Solid fraction on the half-open box (x0, y0, z0, x1, y1, z1); s is indexed
        [z][y][x] over the box. box=None clears the field."""
        if box is None:
            self._call(lib().wt_set_solid_fraction, None, None)
            self._sbox = None
            return
        b = (C.c_int * 6)(*[int(v) for v in box])
        a = np.ascontiguousarray(s, np.float64).ravel()
        self._call(lib().wt_set_solid_fraction, b, _dptr(a))
        self._sbox = tuple(int(v) for v in box)

    def adjoint(self, nsteps: int, window: int, component: int = 0, checkpoint: int = 0,
                keep: bool = False):
        """(J, dJ/ds as [z][y][x] over the box, stats): J is the mean force component
        over the last `window` of `nsteps` steps from the current state. keep leaves
        the run's device memory in the lattice for the next call (an optimisation
        loop); a call without it frees that memory."""
        x0, y0, z0, x1, y1, z1 = self._sbox
        g = np.empty((z1 - z0, y1 - y0, x1 - x0), np.float64)
        cfg = W.wt_adj_cfg(int(nsteps), int(window), int(component), int(checkpoint),
                           int(bool(keep)))
        st = W.wt_adj_stats()
        self._call(lib().wt_adjoint, C.byref(cfg), _dptr(g), C.byref(st))
        self._fields_at = -1
        stats = {k: getattr(st, k) for k, _ in W.wt_adj_stats._fields_}
        return st.J, g, stats

    # ---- checkpoint ------------------------------------------------------------------------
    def get_state(self) -> bytes:
        size = C.c_size_t()
        self._call(lib().wt_state_size, C.byref(size))
        buf = (C.c_char * size.value)()
        self._call(lib().wt_get_state, buf, size.value)
        return bytes(buf)

    def set_state(self, blob: bytes) -> None:
        buf = C.create_string_buffer(blob, len(blob))
        self._call(lib().wt_set_state, buf, len(blob))
        self._fields_at = -1

    # ---- sampling (js/lbm.js:515-545) ------------------------------------------------------
    def sample(self, x: float, y: float, z: float, out=None):
        v = self.sample_points(np.array([[x, y, z]], np.float64))[0]
        if out is None:
            return [float(v[0]), float(v[1]), float(v[2])]
        out[0], out[1], out[2] = float(v[0]), float(v[1]), float(v[2])
        return out

    def sample_points(self, xyz: np.ndarray) -> np.ndarray:
        p = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        out = np.empty_like(p)
        self._call(lib().wt_sample, _dptr(p), p.shape[0], _dptr(out))
        return out

    def isSolid(self, x: float, y: float, z: float) -> bool:
        v = C.c_int()
        self._call(lib().wt_is_solid, float(x), float(y), float(z), C.byref(v))
        return bool(v.value)

    def idx(self, x: int, y: int, z: int) -> int:
        return x + self.nx * (y + self.ny * z)

    # ---- plumbing ----------------------------------------------------------------------------
    @property
    def stream(self) -> int:
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        self._call(lib().wt_get_stream, C.byref(s))
        return s.value or 0

    @property
    def launch_count(self) -> int:
        c = C.c_int64()
        self._call(lib().wt_get_launch_count, C.byref(c))
        return c.value


def _evaluate_inside(inside, X: np.ndarray, Y: np.ndarray, Z: np.ndarray) -> np.ndarray:
    """inside() at every point: one vectorised call when it accepts arrays, else a loop."""
    if X.size == 0:
        return np.zeros(0, np.uint8)
    try:
        r = inside(X, Y, Z)
        r = np.asarray(r)
        if r.shape == X.shape:
            return r.astype(bool).astype(np.uint8)
    except Exception:
        pass
    return np.fromiter((1 if inside(float(x), float(y), float(z)) else 0
                        for x, y, z in zip(X, Y, Z)), np.uint8, X.size)


def sphere_inside(cx: float, cy: float, cz: float, r: float) -> Callable:
    """The analytic sphere point test ||(x,y,z) - c||^2 <= r^2 (vectorised)."""
    r2 = r * r

    def inside(x, y, z):
        dx, dy, dz = x - cx, y - cy, z - cz
        return dx * dx + dy * dy + dz * dz <= r2
    return inside


def sphere_box(cx: float, cy: float, cz: float, r: float, margin: float = 2.0) -> dict:
    return {"x0": cx - r - margin, "y0": cy - r - margin, "z0": cz - r - margin,
            "x1": cx + r + margin, "y1": cy + r + margin, "z1": cz + r + margin}
