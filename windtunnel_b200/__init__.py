"""windtunnel_b200 — B200-native D3Q19 lattice-Boltzmann step of windtunnel.

The compute path is libwt.so (CUDA for sm_100a, C ABI in include/wt.h);
this package holds its host mirror of the reference solver interface.
"""
from ._lib import WTError, lib  # noqa: F401
from .lbm import LBM, sphere_box, sphere_inside  # noqa: F401

__all__ = ["LBM", "WTError", "lib", "sphere_box", "sphere_inside"]
