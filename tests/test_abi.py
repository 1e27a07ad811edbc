"""The C-ABI libraries load without a GPU and export every function that include/*.h
declares; host-side entry points behave (no GPU compute is called here)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from pmdd_b200 import _native

HEADERS = [os.path.join(ROOT, "include", h) for h in ("pmdd.h", "pmdd_host.h")]


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = set()
    for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_ \*]*?)\b(pmdd_[a-z0-9_]+)\s*\(", text):
        names.add(m.group(2))
    return names


def test_headers_declare_functions():
    assert "pmdd_enumerate" in declared_functions(HEADERS[0])
    assert "pmdd_build_from_file" in declared_functions(HEADERS[1])


@pytest.mark.parametrize("header,lib", [("pmdd.h", "libpmdd_gpu.so"), ("pmdd_host.h", "libpmdd_host.so")])
def test_library_exports_every_declared_symbol(header, lib):
    path = os.path.join(_native.LIB_DIR, lib)
    assert os.path.exists(path), f"{lib} not built"
    handle = ctypes.CDLL(path)
    missing = [n for n in sorted(declared_functions(os.path.join(ROOT, "include", header))) if not hasattr(handle, n)]
    assert not missing, missing


def test_python_bindings_cover_headers():
    gpu = declared_functions(HEADERS[0])
    host = declared_functions(HEADERS[1])
    assert gpu <= set(_native.GPU_SYMBOLS), gpu - set(_native.GPU_SYMBOLS)
    assert host <= set(_native.HOST_SYMBOLS), host - set(_native.HOST_SYMBOLS)


def test_struct_sizes_match_c_layout():
    # pmdd_dd: 5 int32 + pad + 7 pointers + 2 int32; pmdd_options: 4 int32 + 2 int64 + 2 int32
    assert ctypes.sizeof(_native.PmddDD) == 5 * 4 + 4 + 7 * 8 + 2 * 4
    assert ctypes.sizeof(_native.PmddOptions) == 40
    assert ctypes.sizeof(_native.PmddFrontier) == 24


def test_options_default_matches_reference_cli_defaults():
    o = _native.PmddOptions()
    _native.gpu_lib().pmdd_options_default(ctypes.byref(o))
    assert (o.method, o.maximization, o.max_cand, o.max_prod, o.device) == (1, 1, 20_000_000, 625_000, 0)
    assert _native.gpu_lib().pmdd_version().startswith(b"pmdd_b200")


def test_sort_points_lex_ascending():
    rng = np.random.default_rng(3)
    pts = rng.integers(-5, 5, size=(200, 4)).astype(np.int32)
    want = pts[np.lexsort(pts.T[::-1])]
    buf = np.ascontiguousarray(pts.copy())
    _native.host_lib().pmdd_sort_points_lex_ascending(buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), 200, 4)
    assert np.array_equal(buf, want)


def test_enumerate_rejects_null_dd_without_gpu_work():
    err = ctypes.create_string_buffer(256)
    rc = _native.gpu_lib().pmdd_enumerate(None, None, None, None, err, len(err))
    assert rc == 1 and b"NULL" in err.value
