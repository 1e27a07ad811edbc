"""TEST INFRASTRUCTURE ONLY -- the oracle.

Python access to (a) the C restatement of the reference's CPU enumeration
(oracle/pmdd_oracle.c, built into oracle/_build/liboracle.so) and (b) the reference's
own CPU binaries built from its sources by oracle/Makefile into oracle/_ref/.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs may
use this package, and only as the checker or the reported CPU baseline.
"""
from __future__ import annotations

import ctypes
import gzip
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


class OracleStats(ctypes.Structure):
    _fields_ = [
        ("candidates_total", ctypes.c_int64),
        ("survivors_total", ctypes.c_int64),
        ("dominance_filtered_total", ctypes.c_int64),
        ("join_products_total", ctypes.c_int64),
        ("layer_coupling", ctypes.c_int32),
        ("pad", ctypes.c_int32),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle restatement`")
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        for name in ("oracle_topdown",):
            getattr(_lib, name).argtypes = [ctypes.c_void_p, ctypes.c_int, P(P(ctypes.c_int32)), P(ctypes.c_int64),
                                            P(OracleStats)]
        _lib.oracle_coupled.argtypes = [ctypes.c_void_p, ctypes.c_int, P(P(ctypes.c_int32)), P(ctypes.c_int64),
                                        P(OracleStats)]
        _lib.oracle_bottomup.argtypes = [ctypes.c_void_p, P(P(ctypes.c_int32)), P(ctypes.c_int64)]
        _lib.oracle_nd_keep.argtypes = [P(ctypes.c_int32), ctypes.c_int64, ctypes.c_int, P(ctypes.c_uint8)]
        _lib.oracle_free.argtypes = [ctypes.c_void_p]
        for name in ("oracle_topdown", "oracle_coupled", "oracle_bottomup"):
            getattr(_lib, name).restype = ctypes.c_int
    return _lib


def _take(ptr, n, d):
    if n == 0:
        lib().oracle_free(ptr)
        return np.zeros((0, d), dtype=np.int32)
    arr = np.ctypeslib.as_array(ptr, shape=(n * d,)).reshape(n, d).copy()
    lib().oracle_free(ptr)
    return arr


def enumerate(dd, method: int = 1, state_dominance: int = 0, stats: dict | None = None) -> np.ndarray:
    """Frontier of a pmdd_b200.DecisionDiagram by the C restatement (methods 1, 2, 3)."""
    view = dd.view
    out = ctypes.POINTER(ctypes.c_int32)()
    n = ctypes.c_int64()
    st = OracleStats()
    if method == 1:
        rc = lib().oracle_topdown(ctypes.addressof(view), state_dominance, ctypes.byref(out), ctypes.byref(n),
                                  ctypes.byref(st))
    elif method == 2:
        rc = lib().oracle_bottomup(ctypes.addressof(view), ctypes.byref(out), ctypes.byref(n))
    elif method == 3:
        rc = lib().oracle_coupled(ctypes.addressof(view), state_dominance, ctypes.byref(out), ctypes.byref(n),
                                  ctypes.byref(st))
    else:
        raise ValueError("method must be 1, 2 or 3")
    if rc != 0:
        raise RuntimeError(f"oracle failed with status {rc}")
    if stats is not None:
        stats.update({name: getattr(st, name) for name, _ in st._fields_ if name != "pad"})
    return _take(out, n.value, view.nobjs)


def nd_keep(points: np.ndarray) -> np.ndarray:
    """Keep flags of the GPU filter rule (first duplicate kept) over one segment."""
    pts = np.ascontiguousarray(points, dtype=np.int32)
    keep = np.zeros(pts.shape[0], dtype=np.uint8)
    lib().oracle_nd_keep(pts.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), pts.shape[0], pts.shape[1],
                         keep.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    return keep.astype(bool)


def sorted_set(points: np.ndarray) -> np.ndarray:
    """Canonical form for set comparison: rows sorted ascending lexicographically."""
    pts = np.asarray(points)
    if pts.shape[0] <= 1:
        return pts.copy()
    return pts[np.lexsort(pts.T[::-1])]


# ------------------------------------------------------- the reference's own binary
def ref_binary(nobjs: int) -> str:
    return os.path.join(REF_DIR, f"multiobj_nobjs{nobjs}")


def have_ref(nobjs: int) -> bool:
    return os.path.exists(ref_binary(nobjs))


def run_ref(path: str, problem_type: int, method: int, nobjs: int, threads: int = 1, state_dominance: int = 0,
            timeout: float = 600.0) -> dict:
    """Runs the reference CPU binary on an instance file; returns its frontier (sorted),
    stdout lines and stats JSONL record."""
    with tempfile.TemporaryDirectory() as td:
        fout = os.path.join(td, "f.csv.gz")
        sout = os.path.join(td, "s.jsonl")
        cmd = [ref_binary(nobjs), path, str(problem_type), str(method), str(state_dominance), "--backend", "cpu",
               "--cpu-threads", str(threads), "--frontier-out", fout, "--stats-out", sout]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference run failed: {' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
        with gzip.open(fout, "rt") as f:
            rows = [list(map(int, line.split(","))) for line in f if line.strip()]
        with open(sout) as f:
            stats = json.loads(f.readline())
    pts = np.array(rows, dtype=np.int64).reshape(-1, nobjs)
    return {"frontier": pts, "stdout": p.stdout.splitlines(), "stats": stats}


def write_flat_dd(dd, path: str) -> None:
    """Writes a pmdd_b200.DecisionDiagram in the file layout oracle/ref_harness.cpp reads."""
    v = dd.view
    a = dd.arrays()
    minw = a["min_weight"]
    st = a["node_state"]
    hdr = np.array([0x46444450, v.nobjs, v.num_layers, v.num_nodes, v.num_arcs, v.num_weights,
                    1 if minw is not None else 0, v.state_words if st is not None else 0], dtype="<i4")
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        for k in ("layer_offsets", "in_arc_offsets", "arc_src", "arc_weight", "weights"):
            f.write(np.ascontiguousarray(a[k], dtype="<i4").tobytes())
        if minw is not None:
            f.write(np.ascontiguousarray(minw, dtype="<i4").tobytes())
        if st is not None:
            f.write(np.ascontiguousarray(st, dtype="<u8").tobytes())


def harness_binary(nobjs: int) -> str:
    return os.path.join(REF_DIR, f"ref_harness_nobjs{nobjs}")


def have_harness(nobjs: int) -> bool:
    return os.path.exists(harness_binary(nobjs))


def run_harness(dd, problem_type: int, method: int, state_dominance: int = 0, timeout: float = 600.0) -> dict:
    """The reference's CPU enumeration (methods 1 and 3, with its state-dominance passes)
    run on this DD in this project's node numbering; returns its counters and frontier."""
    nobjs = dd.view.nobjs
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "dd.bin")
        write_flat_dd(dd, path)
        cmd = [harness_binary(nobjs), path, str(problem_type), str(method), str(state_dominance)]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"reference harness failed: {' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
    lines = p.stdout.splitlines()
    stats = json.loads(lines[0])
    rows = [list(map(int, line.split(","))) for line in lines[1:] if line.strip()]
    return {"frontier": np.array(rows, dtype=np.int64).reshape(-1, nobjs), "stats": stats}
