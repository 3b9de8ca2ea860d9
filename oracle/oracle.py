"""ctypes binding of the CPU oracle (lbm_oracle.c) — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
use this module, and only as the checker. `OracleLBM` restates js/lbm.js
(float32 storage = the reference's own arithmetic; float64 storage = the
FP64 oracle) with the same interface as windtunnel_b200.LBM.

Build: `python -m oracle.build` (gcc -O2 -ffp-contract=off -fopenmp).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liblbm_oracle.so"
SOURCES = [HERE / "lbm_oracle.c", HERE / "lbm_oracle_impl.h", HERE.parent / "include" / "wt.h"]


def build(force: bool = False) -> Path:
    """Compile liblbm_oracle.so next to its sources when they changed."""
    if not force and LIB_PATH.exists():
        t = LIB_PATH.stat().st_mtime
        if all(s.stat().st_mtime <= t for s in SOURCES):
            return LIB_PATH
    cmd = ["gcc", "-O2", "-std=c11", "-Wall", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           "-fPIC", "-shared", "-o", str(LIB_PATH), str(HERE / "lbm_oracle.c"), "-lm"]
    subprocess.run(cmd, check=True)
    return LIB_PATH


class wt_params(C.Structure):
    _fields_ = [
        ("u0", C.c_double), ("tau", C.c_double), ("les", C.c_int32), ("trt", C.c_int32),
        ("csm", C.c_double), ("lambda_", C.c_double), ("moving_walls", C.c_int32),
        ("side_bc", C.c_int32), ("math", C.c_int32), ("kernel", C.c_int32),
        ("f16_rounding", C.c_int32), ("reserved", C.c_int32),
    ]


class wt_body_stats(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("frontal_area", "planform_area", "solid_cells",
                                         "ride_height", "ground", "moving_walls")]


_lib = None
_D = C.POINTER(C.c_double)
_U8 = C.POINTER(C.c_uint8)
_F = C.POINTER(C.c_float)


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    L = C.CDLL(str(LIB_PATH))
    for pfx in ("or32_", "or64_"):
        sig = {
            "create": ([C.c_int] * 3, C.c_void_p),
            "destroy": ([C.c_void_p], None),
            "set_params": ([C.c_void_p, C.POINTER(wt_params)], None),
            "get_params": ([C.c_void_p, C.POINTER(wt_params)], None),
            "reset": ([C.c_void_p], C.c_int),
            "init_eq_noise": ([C.c_void_p, C.c_uint64, C.c_double], C.c_int),
            "voxelize_mask": ([C.c_void_p, _D, _U8, C.c_size_t, _U8, _D, C.c_int, C.c_double],
                              C.c_int),
            "step": ([C.c_void_p, C.c_int, _D, C.c_int], C.c_int),
            "get_force": ([C.c_void_p, _D], None),
            "get_fields": ([C.c_void_p, _F, _F, _F, _F], None),
            "get_solid": ([C.c_void_p, _U8], None),
            "get_near": ([C.c_void_p, _U8], None),
            "get_pop": ([C.c_void_p, C.c_int, _D], None),
            "get_pop_raw": ([C.c_void_p, C.c_int, C.c_void_p], None),
            "set_pop_raw": ([C.c_void_p, C.c_int, C.c_void_p], None),
            "get_body_stats": ([C.c_void_p, C.POINTER(wt_body_stats)], None),
            "get_steps": ([C.c_void_p], C.c_long),
            "get_parity": ([C.c_void_p], C.c_int),
            "sample": ([C.c_void_p, C.c_double, C.c_double, C.c_double, _D], None),
            "is_solid": ([C.c_void_p, C.c_double, C.c_double, C.c_double], C.c_int),
            "step_sample": ([C.c_void_p, C.c_int, C.c_int, C.c_int], C.c_long),
            "set_solid_fraction": ([C.c_void_p, C.POINTER(C.c_int), _D], C.c_int),
            "adjoint": ([C.c_void_p, C.c_int, C.c_int, C.c_int, _D, _D], C.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, pfx + name)
            fn.argtypes = args
            fn.restype = res
    L.or_default_params.argtypes = [C.POINTER(wt_params)]
    L.or_default_params.restype = None
    L.or_voxel_range.argtypes = [C.c_int, C.c_int, C.c_int, _D, C.POINTER(C.c_int)]
    L.or_voxel_range.restype = None
    L.or_lookup_mask.argtypes = [_U8, C.c_int, C.c_int, C.c_int, _D, C.c_double, _D, _D,
                                 C.c_double, C.c_int, C.c_int, C.c_int, _D, _U8]
    L.or_lookup_mask.restype = C.c_long
    L.or_voxel_dims.argtypes = [_F, C.c_long, C.c_int, C.c_void_p]
    L.or_voxel_dims.restype = C.c_int
    L.or_voxel_build.argtypes = [_F, C.c_long, C.c_int, _U8, C.c_void_p]
    L.or_voxel_build.restype = C.c_int
    L.or_uniform_draw.argtypes = [C.c_uint64, C.c_uint64]
    L.or_uniform_draw.restype = C.c_double
    L.or_toint32_export.argtypes = [C.c_double]
    L.or_toint32_export.restype = C.c_int32
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(_D)


def _box6(box) -> np.ndarray:
    if isinstance(box, dict):
        v = [box[k] for k in ("x0", "y0", "z0", "x1", "y1", "z1")]
    else:
        v = list(box)
    return np.ascontiguousarray(v, np.float64)


def voxel_range(nx, ny, nz, box) -> tuple:
    rg = (C.c_int * 6)()
    lib().or_voxel_range(nx, ny, nz, _dp(_box6(box)), rg)
    return tuple(rg)


def lookup_mask(grid, gmin, ginv, M, P, scale, nx, ny, nz, box) -> np.ndarray:
    """js/shapes.js:369-388 evaluated at the cell centres of box's scan range."""
    g = np.ascontiguousarray(grid, np.uint8)
    gnz, gny, gnx = g.shape
    x0, x1, y0, y1, z0, z1 = voxel_range(nx, ny, nz, box)
    cnt = max(0, x1 - x0 + 1) * max(0, y1 - y0 + 1) * max(0, z1 - z0 + 1)
    out = np.zeros(cnt, np.uint8)
    lib().or_lookup_mask(g.ctypes.data_as(_U8), gnx, gny, gnz,
                         _dp(np.ascontiguousarray(gmin, np.float64)), float(ginv),
                         _dp(np.ascontiguousarray(M, np.float64)),
                         _dp(np.ascontiguousarray(P, np.float64)), float(scale), nx, ny, nz,
                         _dp(_box6(box)), out.ctypes.data_as(_U8))
    return out


class or_voxel_info(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("tris", C.c_int),
                ("cell", C.c_double), ("inv", C.c_double), ("min", C.c_double * 3),
                ("ext", C.c_double * 3), ("centre", C.c_double * 3), ("bbox", C.c_double * 6),
                ("solid", C.c_long), ("openness", C.c_double)]


def voxel_build(P, res: int = 96):
    """Voxel.build (js/voxel.js:48-102): (grid [nz][ny][nx] uint8, info dict)."""
    L = lib()
    p = np.ascontiguousarray(P, np.float32).ravel()
    ntri = p.size // 9
    vi = or_voxel_info()
    rc = L.or_voxel_dims(p.ctypes.data_as(_F), ntri, int(res), C.byref(vi))
    if rc:
        raise ValueError({-1: "Mesh has no triangles.", -2: "Mesh is degenerate (zero size).",
                          -3: "Voxel grid too large; lower the resolution."}.get(rc, rc))
    grid = np.zeros((vi.nz, vi.ny, vi.nx), np.uint8)
    rc = L.or_voxel_build(p.ctypes.data_as(_F), ntri, int(res), grid.ctypes.data_as(_U8),
                          C.byref(vi))
    if rc:
        raise ValueError(f"oracle voxel build failed ({rc})")
    info = {k: (list(getattr(vi, k)) if k in ("min", "ext", "centre", "bbox") else
                getattr(vi, k)) for k, _ in or_voxel_info._fields_}
    return grid, info


def uniform_draw(seed: int, k: int) -> float:
    return lib().or_uniform_draw(C.c_uint64(seed), C.c_uint64(k))


class OracleLBM:
    """The reference solver restated on the CPU (storage 'f32' or 'f64')."""

    def __init__(self, nx, ny, nz, storage: str = "f32", side_bc: str = "eq"):
        self.L = lib()
        self.pfx = {"f32": "or32_", "f64": "or64_"}[storage]
        self.storage = storage
        self.h = self._fn("create")(nx, ny, nz)
        if not self.h:
            raise ValueError("oracle create failed")
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = nx * ny * nz
        p = self.params()
        p.side_bc = {"eq": 0, "freeslip": 1}[side_bc]
        self._fn("set_params")(self.h, C.byref(p))

    def _fn(self, name):
        return getattr(self.L, self.pfx + name)

    def close(self):
        if self.h:
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> wt_params:
        p = wt_params()
        self._fn("get_params")(self.h, C.byref(p))
        return p

    def set_params(self, **kw):
        p = self.params()
        for k, v in kw.items():
            key = {"lambda": "lambda_", "movingWalls": "moving_walls"}.get(k, k)
            if key == "side_bc" and isinstance(v, str):
                v = {"eq": 0, "freeslip": 1}[v]
            cur = getattr(p, key)
            setattr(p, key, float(v) if isinstance(cur, float) else int(v))
        self._fn("set_params")(self.h, C.byref(p))

    def reset(self):
        self._fn("reset")(self.h)

    def init_eq_noise(self, seed, amp):
        self._fn("init_eq_noise")(self.h, C.c_uint64(seed), float(amp))

    def voxelize_mask(self, box, mask, ground=False, wall_set=None, wall_vel=None, roadVel=0.0):
        m = np.ascontiguousarray(mask, np.uint8).ravel()
        ws = wv = None
        if wall_set is not None:
            ws = np.ascontiguousarray(wall_set, np.uint8).ravel()
            wv = np.ascontiguousarray(wall_vel, np.float64).ravel()
        rc = self._fn("voxelize_mask")(self.h, _dp(_box6(box)), m.ctypes.data_as(_U8), m.size,
                                       ws.ctypes.data_as(_U8) if ws is not None else None,
                                       _dp(wv) if wv is not None else None, int(bool(ground)),
                                       float(roadVel))
        if rc != 0:
            raise ValueError(f"oracle voxelize failed ({rc})")

    def voxelize(self, inside, box, ground=False, wallVel=None, roadVel=0.0):
        from windtunnel_b200.lbm import _evaluate_inside  # host-side closure evaluation only
        x0, x1, y0, y1, z0, z1 = voxel_range(self.nx, self.ny, self.nz, box)
        ex, ey, ez = max(0, x1 - x0 + 1), max(0, y1 - y0 + 1), max(0, z1 - z0 + 1)
        zz, yy, xx = np.meshgrid(np.arange(z0, z0 + ez) + 0.5, np.arange(y0, y0 + ey) + 0.5,
                                 np.arange(x0, x0 + ex) + 0.5, indexing="ij")
        X, Y, Z = xx.ravel(), yy.ravel(), zz.ravel()
        mask = _evaluate_inside(inside, X, Y, Z)
        ws = wv = None
        if wallVel is not None:
            ws = np.zeros(mask.size, np.uint8)
            wv = np.zeros((mask.size, 3), np.float64)
            out = [0.0, 0.0, 0.0]
            for m in np.flatnonzero(mask):
                if wallVel(float(X[m]), float(Y[m]), float(Z[m]), out):
                    ws[m] = 1
                    wv[m] = out
        self.voxelize_mask(box, mask, ground, ws, wv, roadVel)

    def step(self):
        self._fn("step")(self.h, 1, None, 1)

    def step_forces(self, n: int, threads: int = 1) -> np.ndarray:
        out = np.empty(3 * n, np.float64)
        if n > 0:
            self._fn("step")(self.h, n, _dp(out), int(threads))
        return out.reshape(n, 3)

    def step_sample(self, z0: int, z1: int, threads: int) -> int:
        """One step's work on interior planes [z0, z1) only (buffers not flipped)."""
        return self._fn("step_sample")(self.h, z0, z1, int(threads))

    @property
    def force(self):
        out = np.empty(3, np.float64)
        self._fn("get_force")(self.h, _dp(out))
        return out

    def fields(self):
        a = [np.empty(self.n, np.float32) for _ in range(4)]
        self._fn("get_fields")(self.h, *[x.ctypes.data_as(_F) for x in a])
        return tuple(a)

    @property
    def solid(self):
        out = np.empty(self.n, np.uint8)
        self._fn("get_solid")(self.h, out.ctypes.data_as(_U8))
        return out

    @property
    def near(self):
        out = np.empty(self.n, np.uint8)
        self._fn("get_near")(self.h, out.ctypes.data_as(_U8))
        return out

    def populations(self, which="f", dtype="f64"):
        if dtype == "raw":
            npd = np.float32 if self.storage == "f32" else np.float64
            out = np.empty(19 * self.n, npd)
            self._fn("get_pop_raw")(self.h, 0 if which == "f" else 1, out.ctypes.data)
            return out.reshape(19, self.n)
        out = np.empty(19 * self.n, np.float64)
        self._fn("get_pop")(self.h, 0 if which == "f" else 1, _dp(out))
        out = out.reshape(19, self.n)
        return out.astype(np.float32) if dtype == "f32" else out

    def set_populations_raw(self, data, which="f"):
        npd = np.float32 if self.storage == "f32" else np.float64
        a = np.ascontiguousarray(data, npd)
        self._fn("set_pop_raw")(self.h, 0 if which == "f" else 1, a.ctypes.data)

    def body_stats(self) -> wt_body_stats:
        s = wt_body_stats()
        self._fn("get_body_stats")(self.h, C.byref(s))
        return s

    @property
    def steps(self):
        return self._fn("get_steps")(self.h)

    @property
    def parity(self):
        return self._fn("get_parity")(self.h)

    def sample(self, x, y, z):
        out = np.empty(3, np.float64)
        self._fn("sample")(self.h, x, y, z, _dp(out))
        return out

    def isSolid(self, x, y, z):
        return bool(self._fn("is_solid")(self.h, x, y, z))

    # partial bounce-back and its adjoint (no reference counterpart)
    def set_solid_fraction(self, box, s):
        """box = (x0, y0, z0, x1, y1, z1), half-open; s indexed [z][y][x] over the box."""
        b = (C.c_int * 6)(*[int(v) for v in box])
        a = np.ascontiguousarray(s, np.float64).ravel()
        self._sbox = tuple(int(v) for v in box)
        rc = self._fn("set_solid_fraction")(self.h, b, _dp(a))
        if rc != 0:
            raise ValueError(f"oracle set_solid_fraction failed ({rc})")

    def adjoint(self, nsteps: int, window: int, comp: int = 0):
        """(J, dJ/ds over the box as [z][y][x]); the lattice advances nsteps."""
        x0, y0, z0, x1, y1, z1 = self._sbox
        g = np.empty((z1 - z0, y1 - y0, x1 - x0), np.float64)
        J = C.c_double()
        rc = self._fn("adjoint")(self.h, nsteps, window, comp, C.byref(J), _dp(g))
        if rc != 0:
            raise ValueError(f"oracle adjoint failed ({rc})")
        return J.value, g
