"""The C-ABI library loads and exports every entry point declared in
include/*.h; argument errors come back as status codes (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

from yaoray_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(yrc_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_device_probe_never_fault():
    L = _lib.lib()
    assert L.yrc_version().decode() == "0.1.0"
    assert L.yrc_device_available() in (0, 1)


def test_null_arguments_return_invalid_argument():
    L = _lib.lib()
    assert L.yrc_bvh_build(None, None, None) == _lib.YRC_ERR_INVALID_ARGUMENT
    assert "null" in L.yrc_last_error().decode()
    assert L.yrc_accel_create_flat(None, None, None) == _lib.YRC_ERR_INVALID_ARGUMENT
    assert L.yrc_trace_host(None, None, 0, 0, None, None, None, None) == _lib.YRC_ERR_INVALID_ARGUMENT
    assert L.yrc_trace_device(None, None, 0, 0, None, None, None, None) == _lib.YRC_ERR_INVALID_ARGUMENT
    assert L.yrc_probe_device(None, None, None, 0, None, None, None, None, None) == _lib.YRC_ERR_INVALID_ARGUMENT


def test_bad_geometry_rejected_before_any_device_work():
    L = _lib.lib()
    g = _lib.Geometry()
    g.vertex_count = 3
    g.positions = None  # non-zero count with a null array
    v = _lib.BvhView()
    h = C.c_void_p()
    assert L.yrc_accel_create_flat(C.byref(g), C.byref(v), C.byref(h)) == _lib.YRC_ERR_INVALID_ARGUMENT
    assert "null geometry array" in L.yrc_last_error().decode()


def test_struct_sizes_match_header():
    assert _lib.NODE_DTYPE.itemsize == 32
    assert C.sizeof(_lib.PreparedInstance) == 4 * (2 + 16 + 16 + 6)
    assert np.dtype(_lib.RAY_DTYPE).itemsize == 32 and np.dtype(_lib.HIT_DTYPE).itemsize == 16
