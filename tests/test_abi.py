"""The C ABI: libwt.so loads and exports every entry point include/wt.h declares.

No compute call is made here (these run without a GPU).
"""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "wt.h"


def declared_functions(header: Path) -> list[str]:
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wt_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions(HEADER)
    for required in ("wt_create", "wt_destroy", "wt_step", "wt_voxelize_mask", "wt_voxelize_grid",
                     "wt_get_fields", "wt_get_populations", "wt_last_error", "wt_get_state",
                     "wt_set_state", "wt_sample", "wt_is_solid", "wt_reset"):
        assert required in names


def test_library_exports_every_declared_symbol(wt_lib):
    missing = [n for n in declared_functions(HEADER) if not hasattr(wt_lib, n)]
    assert not missing, f"not exported: {missing}"


def test_exports_are_c_symbols(wt_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", wt_lib._name], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (wt_[a-z0-9_]+)\b", out))
    assert set(declared_functions(HEADER)) <= exported


def test_default_params_match_reference(wt_lib):
    """js/lbm.js:106-111 defaults, without touching a device."""
    from windtunnel_b200 import _lib
    p = _lib.default_params()
    assert p.u0 == 0.06 and p.tau == 0.5035 and p.les == 1 and p.csm == 0.14
    assert p.trt == 1 and p.lambda_ == 0.25 and p.side_bc == 0 and p.math == 0
    assert p.kernel == 0 and p.f16_rounding == 0 and p.reserved == 0


def test_create_rejects_bad_dims_on_host(wt_lib):
    """Argument checks happen before any CUDA call."""
    from windtunnel_b200 import _lib
    h = ctypes.c_void_p()
    assert wt_lib.wt_create(2, 8, 8, 0, ctypes.byref(h)) == _lib.WT_ERR_ARG
    assert b"at least 3" in wt_lib.wt_last_error(None)
    assert wt_lib.wt_create(8, 8, 8, 7, ctypes.byref(h)) == _lib.WT_ERR_ARG
    assert wt_lib.wt_create(8, 8, 8, 0, None) == _lib.WT_ERR_ARG
    assert h.value is None


def test_null_handle_is_an_argument_error(wt_lib):
    from windtunnel_b200 import _lib
    assert wt_lib.wt_step(None, 1, None) == _lib.WT_ERR_ARG
    assert wt_lib.wt_reset(None) == _lib.WT_ERR_ARG
    assert wt_lib.wt_destroy(None) == _lib.WT_OK


def test_binding_constants_match_the_header():
    """Every WT_* enumerator of include/wt.h has the same value in the ctypes
    binding (a drifted constant would select the wrong kernel or storage)."""
    import re

    from windtunnel_b200 import _lib as W
    text = (ROOT / "include" / "wt.h").read_text()
    body = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    found = dict(re.findall(r"\b(WT_[A-Z0-9_]+)\s*=\s*(-?\d+)", body))
    assert len(found) > 20
    for name, value in found.items():
        assert hasattr(W, name), name
        assert getattr(W, name) == int(value), name


def test_binding_structs_match_the_header(tmp_path):
    """The ctypes structs have the C layout of include/wt.h (sizes and field
    offsets, compiled with the host C compiler)."""
    import ctypes
    import shutil
    import subprocess

    from windtunnel_b200 import _lib as W
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    structs = ["wt_params", "wt_body_stats", "wt_adj_cfg", "wt_adj_stats", "wt_voxel_info"]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "wt.h"', "int main(void) {"]
    for s in structs:
        lines.append(f'  printf("{s} %zu\\n", sizeof({s}));')
        for f, _ in getattr(W, s)._fields_:
            cf = f[:-1] if f.endswith("_") else f   # lambda_ is the C field lambda
            lines.append(f'  printf("{s}.{f} %zu\\n", offsetof({s}, {cf}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True,
                                                        text=True, check=True).stdout.split("\n") if l)
    for s in structs:
        cls = getattr(W, s)
        assert int(out[s]) == ctypes.sizeof(cls), s
        for f, _ in cls._fields_:
            assert int(out[f"{s}.{f}"]) == getattr(cls, f).offset, (s, f)
