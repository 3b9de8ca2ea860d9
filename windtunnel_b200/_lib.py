"""ctypes binding of libwt.so — the C ABI declared in include/wt.h.

The library is loaded from this package directory (built in-tree by
windtunnel_b200.build). There is no fallback: if the shared object is
missing or cannot be loaded, `lib()` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libwt.so"

WT_OK = 0
WT_ERR_ARG = -1
WT_ERR_OOM = -2
WT_ERR_CUDA = -3
WT_ERR_DIVERGED = -4
WT_ERR_TIMEOUT = -5
WT_ERR_STATE = -6
WT_ERR_UNSUPPORTED = -7

WT_STORE_F32 = 0
WT_STORE_F16DEV = 1
WT_STORE_F64 = 2
WT_F16_SCALE = 4096.0

WT_MATH_FAST = 0
WT_MATH_EXACT = 1

WT_SIDE_EQ = 0
WT_SIDE_FREESLIP = 1

WT_KERNEL_AUTO = 0
WT_KERNEL_DIRECT = 1
WT_KERNEL_LEAN = 7
WT_KERNEL_PAIR = 8

WT_ROUND_NEAREST = 0
WT_ROUND_STOCHASTIC = 1

WT_FLUID = 0
WT_SOLID_OBJ = 1
WT_SOLID_WALL = 2

WT_BUF_F = 0
WT_BUF_G = 1

ERROR_NAMES = {
    WT_ERR_ARG: "WT_ERR_ARG",
    WT_ERR_OOM: "WT_ERR_OOM",
    WT_ERR_CUDA: "WT_ERR_CUDA",
    WT_ERR_DIVERGED: "WT_ERR_DIVERGED",
    WT_ERR_TIMEOUT: "WT_ERR_TIMEOUT",
    WT_ERR_STATE: "WT_ERR_STATE",
    WT_ERR_UNSUPPORTED: "WT_ERR_UNSUPPORTED",
}


class wt_params(C.Structure):
    _fields_ = [
        ("u0", C.c_double),
        ("tau", C.c_double),
        ("les", C.c_int32),
        ("trt", C.c_int32),
        ("csm", C.c_double),
        ("lambda_", C.c_double),
        ("moving_walls", C.c_int32),
        ("side_bc", C.c_int32),
        ("math", C.c_int32),
        ("kernel", C.c_int32),
        ("f16_rounding", C.c_int32),
        ("reserved", C.c_int32),
    ]


class wt_body_stats(C.Structure):
    _fields_ = [
        ("frontal_area", C.c_int32),
        ("planform_area", C.c_int32),
        ("solid_cells", C.c_int32),
        ("ride_height", C.c_int32),
        ("ground", C.c_int32),
        ("moving_walls", C.c_int32),
    ]


class wt_adj_cfg(C.Structure):
    _fields_ = [("nsteps", C.c_int32), ("window", C.c_int32), ("component", C.c_int32),
                ("checkpoint", C.c_int32), ("keep", C.c_int32), ("reserved", C.c_int32 * 3)]


class wt_adj_stats(C.Structure):
    _fields_ = [("J", C.c_double), ("forward_ms", C.c_double), ("backward_ms", C.c_double),
                ("device_bytes", C.c_int64), ("checkpoints", C.c_int32), ("segment", C.c_int32)]


class wt_voxel_info(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("reserved", C.c_int32),
                ("tris", C.c_int64), ("cell", C.c_double), ("inv", C.c_double),
                ("min", C.c_double * 3), ("ext", C.c_double * 3), ("centre", C.c_double * 3),
                ("bbox", C.c_double * 6), ("solid", C.c_int64), ("openness", C.c_double)]


class WTError(RuntimeError):
    """A wt_* call returned a negative status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_U8 = C.POINTER(C.c_uint8)
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)

# name -> argtypes (every function returns int unless listed in _RESTYPES)
SIGNATURES = {
    "wt_default_params": [C.POINTER(wt_params)],
    "wt_create": [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_P)],
    "wt_destroy": [_P],
    "wt_last_error": [_P],
    "wt_get_dims": [_P, _I, _I, _I, _I],
    "wt_set_params": [_P, C.POINTER(wt_params)],
    "wt_get_params": [_P, C.POINTER(wt_params)],
    "wt_reset": [_P],
    "wt_init_eq_noise": [_P, C.c_uint64, C.c_double],
    "wt_voxel_range": [_P, _D, _I],
    "wt_voxelize_mask": [_P, _D, _U8, C.c_size_t, _U8, _D, C.c_int, C.c_double],
    "wt_voxelize_grid": [_P, _U8, C.c_int, C.c_int, C.c_int, _D, C.c_double, _D, _D, C.c_double,
                         _D, C.c_int, C.c_double],
    "wt_get_body_stats": [_P, C.POINTER(wt_body_stats)],
    "wt_step": [_P, C.c_int, _D],
    "wt_step_noalloc": [_P, C.c_int, _D],
    "wt_get_force": [_P, _D],
    "wt_get_steps": [_P, C.POINTER(C.c_int64), _I],
    "wt_get_fields": [_P, _F, _F, _F, _F],
    "wt_get_solid": [_P, _U8],
    "wt_get_near": [_P, _U8],
    "wt_get_populations": [_P, C.c_int, C.c_int, C.c_void_p, C.c_size_t],
    "wt_set_populations": [_P, C.c_int, C.c_int, C.c_void_p, C.c_size_t],
    "wt_state_size": [_P, C.POINTER(C.c_size_t)],
    "wt_get_state": [_P, C.c_void_p, C.c_size_t],
    "wt_set_state": [_P, C.c_void_p, C.c_size_t],
    "wt_sample": [_P, _D, C.c_int, _D],
    "wt_is_solid": [_P, C.c_double, C.c_double, C.c_double, _I],
    "wt_get_stream": [_P, C.POINTER(_P)],
    "wt_get_launch_count": [_P, C.POINTER(C.c_int64)],
    "wt_set_solid_fraction": [_P, _I, _D],
    "wt_adjoint": [_P, C.POINTER(wt_adj_cfg), _D, C.POINTER(wt_adj_stats)],
    "wt_voxel_dims": [C.POINTER(C.c_float), C.c_int64, C.c_int, C.POINTER(wt_voxel_info)],
    "wt_voxel_build": [C.POINTER(C.c_float), C.c_int64, C.c_int, C.POINTER(C.c_uint8), C.c_size_t,
                       C.POINTER(wt_voxel_info)],
    "wt_voxel_last_error": [],
    "wt_slice": [_P, C.c_int, C.c_int, C.c_int, _F, C.c_size_t],
    "wt_advect": [_P, _D, C.c_int, C.c_double, _U8, _F],
}
_RESTYPES = {"wt_default_params": None, "wt_last_error": C.c_char_p,
             "wt_voxel_last_error": C.c_char_p}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load libwt.so once and declare every prototype; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("WT_LIB", str(LIB_PATH))
    if not Path(path).exists():
        raise RuntimeError(
            f"libwt.so not found at {path}; build it with `python -m windtunnel_b200.build`")
    L = C.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, C.c_int)
    _lib = L
    return L


def check(code: int, handle=None) -> int:
    """Raise WTError for a negative status, with the handle's message."""
    if code >= 0:
        return code
    msg = lib().wt_last_error(handle)
    raise WTError(code, msg.decode() if msg else "")


def default_params() -> wt_params:
    p = wt_params()
    lib().wt_default_params(C.byref(p))
    return p
