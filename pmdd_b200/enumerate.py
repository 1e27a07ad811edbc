"""Python mirror of the reference's GPU enumeration seam.

The reference (src/pmdd/enum/gpu/cuda_wrappers.hpp:11-21) exposes four functions; each
returns a new ParetoFrontier or NULL with *reason set.  Here each returns the frontier
as an (F, nobjs) integer array and raises `CudaEnumerationError` (carrying the reason)
on failure.  `stats`, when given, is a dict updated in place with the GPU fields of
the reference's EnumerationStats.  The frontier comes back unsorted; the reference's
main sorts it afterwards (`sort_lexicographic_ascending`).
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Optional

import numpy as np

from . import _native
from .dd import DecisionDiagram

DEFAULT_MAX_CAND = 20_000_000   # --max-cand default (src/pmdd/util/cli_parser.hpp:10)
DEFAULT_MAX_PROD = 625_000      # --max-prod default (src/pmdd/util/cli_parser.hpp:11)


class CudaEnumerationError(RuntimeError):
    def __init__(self, status: int, reason: str):
        super().__init__(f"GPU enumeration failed ({_native.STATUS_NAMES.get(status, status)}): {reason}")
        self.status = status
        self.reason = reason


def _options(method, problem_type, state_dominance, maximization, max_cand, max_prod, device):
    o = _native.PmddOptions()
    _native.gpu_lib().pmdd_options_default(ctypes.byref(o))
    o.method = method
    o.problem_type = problem_type
    o.state_dominance = state_dominance
    o.maximization = 1 if maximization else 0
    o.max_cand = int(max_cand)
    o.max_prod = int(max_prod)
    o.device = device
    return o


def _to_array(fr: _native.PmddFrontier) -> np.ndarray:
    n, d = fr.num_points, fr.nobjs
    dtype = np.int64 if fr.elem_bytes == 8 else np.int32
    if n == 0 or not fr.points:
        return np.zeros((0, d), dtype=dtype)
    buf = (ctypes.c_char * (n * d * fr.elem_bytes)).from_address(fr.points)
    return np.frombuffer(buf, dtype=dtype).reshape(n, d).copy()


def enumerate_dd(dd: DecisionDiagram, method: int = 1, problem_type: Optional[int] = None,
                 state_dominance: int = 0, maximization: bool = True, max_cand: int = DEFAULT_MAX_CAND,
                 max_prod: int = DEFAULT_MAX_PROD, device: int = 0, stats: Optional[dict] = None) -> np.ndarray:
    """One frontier through pmdd_enumerate (the C ABI)."""
    lib = _native.gpu_lib()
    o = _options(method, problem_type or dd.problem_type, state_dominance, maximization, max_cand, max_prod, device)
    fr = _native.PmddFrontier()
    st = _native.PmddStats()
    err = ctypes.create_string_buffer(512)
    view = dd.view
    rc = lib.pmdd_enumerate(ctypes.byref(view), ctypes.byref(o), ctypes.byref(fr), ctypes.byref(st), err, len(err))
    if rc != _native.PMDD_OK:
        raise CudaEnumerationError(rc, err.value.decode(errors="replace"))
    try:
        out = _to_array(fr)
    finally:
        lib.pmdd_frontier_free(ctypes.byref(fr))
    if stats is not None:
        stats.update(st.as_dict())
    return out


def enumerate_batch(dds: Iterable[DecisionDiagram], method: int = 1, state_dominance: int = 0,
                    max_cand: int = DEFAULT_MAX_CAND, max_prod: int = DEFAULT_MAX_PROD, device: int = 0,
                    stats: Optional[dict] = None) -> list:
    """Frontiers of many DDs, advanced together in shared launches."""
    dds = list(dds)
    lib = _native.gpu_lib()
    n = len(dds)
    views = (_native.PmddDD * max(n, 1))()
    for i, dd in enumerate(dds):
        views[i] = dd.view
    ptype = dds[0].problem_type if dds else 1
    o = _options(method, ptype, state_dominance, True, max_cand, max_prod, device)
    outs = (_native.PmddFrontier * max(n, 1))()
    status = (ctypes.c_int32 * max(n, 1))()
    st = _native.PmddStats()
    err = ctypes.create_string_buffer(512)
    rc = lib.pmdd_enumerate_batch(views, n, ctypes.byref(o), outs, status, ctypes.byref(st), err, len(err))
    try:
        if rc != _native.PMDD_OK:
            raise CudaEnumerationError(rc, err.value.decode(errors="replace"))
        res = [_to_array(outs[i]) for i in range(n)]
    finally:
        for i in range(n):
            lib.pmdd_frontier_free(ctypes.byref(outs[i]))
    if stats is not None:
        stats.update(st.as_dict())
    return res


def pareto_filter(points: np.ndarray, device: int = 0) -> np.ndarray:
    """Maximal points of an (n, d) int32 set under componentwise >= (one copy of each
    group of equal points), computed on the GPU (pmdd_pareto_filter)."""
    pts = np.ascontiguousarray(points, dtype=np.int32)
    n, d = pts.shape
    out = np.empty_like(pts)
    n_out = ctypes.c_int64()
    err = ctypes.create_string_buffer(512)
    P = ctypes.POINTER(ctypes.c_int32)
    rc = _native.gpu_lib().pmdd_pareto_filter(pts.ctypes.data_as(P), n, d, out.ctypes.data_as(P),
                                              ctypes.byref(n_out), device, err, len(err))
    if rc != _native.PMDD_OK:
        raise CudaEnumerationError(rc, err.value.decode(errors="replace"))
    return out[: n_out.value].copy()


class ResidentSet:
    """DDs uploaded once to device memory (pmdd_resident_*); each `enumerate` call runs
    a batch over them with no host->device DD traffic."""

    def __init__(self, dds: Iterable[DecisionDiagram], device: int = 0):
        self.dds = list(dds)
        lib = _native.gpu_lib()
        n = len(self.dds)
        views = (_native.PmddDD * max(n, 1))()
        for i, dd in enumerate(self.dds):
            views[i] = dd.view
        err = ctypes.create_string_buffer(512)
        self._h = lib.pmdd_resident_upload(views, n, device, err, len(err))
        if not self._h:
            raise CudaEnumerationError(3, err.value.decode(errors="replace"))
        self._lib = lib
        self.device = device
        self.count = n
        self.problem_type = self.dds[0].problem_type if self.dds else 1

    @classmethod
    def from_knapsack(cls, instances: Iterable, device: int = 0) -> "ResidentSet":
        """Knapsack BDDs built on the device (pmdd_resident_build_knapsack) from
        (profits (nobjs, n), weights (n,), capacity) triples; only those arrays cross the bus."""
        items = [(np.ascontiguousarray(p, dtype=np.int32), np.ascontiguousarray(w, dtype=np.int32), int(c))
                 for p, w, c in instances]
        n = len(items)
        specs = (_native.PmddKnapsack * max(n, 1))()
        P32 = ctypes.POINTER(ctypes.c_int32)
        for i, (p, w, c) in enumerate(items):
            if p.ndim != 2 or w.ndim != 1 or p.shape[1] != w.shape[0]:
                raise ValueError(f"instance {i}: profits must be (nobjs, n) and weights (n,)")
            specs[i] = _native.PmddKnapsack(w.shape[0], p.shape[0], p.ctypes.data_as(P32), w.ctypes.data_as(P32), c, 0)
        lib = _native.gpu_lib()
        err = ctypes.create_string_buffer(512)
        self = cls.__new__(cls)
        self.dds = []
        self._lib = lib
        self.device = device
        self.count = n
        self.problem_type = 1
        self._h = lib.pmdd_resident_build_knapsack(specs, n, device, err, len(err))
        if not self._h:
            raise CudaEnumerationError(1, err.value.decode(errors="replace"))
        return self

    @classmethod
    def from_tsp(cls, costs: Iterable, device: int = 0) -> "ResidentSet":
        """TSP MDDs on the device (pmdd_resident_build_tsp) from cost matrices
        (nobjs, n, n): the n-city structure is built once on the GPU and shared, each
        instance uploads only its weight table."""
        mats = [np.ascontiguousarray(c, dtype=np.int32) for c in costs]
        n = len(mats)
        specs = (_native.PmddTsp * max(n, 1))()
        P32 = ctypes.POINTER(ctypes.c_int32)
        for i, c in enumerate(mats):
            if c.ndim != 3 or c.shape[1] != c.shape[2]:
                raise ValueError(f"instance {i}: costs must be (nobjs, n, n)")
            specs[i] = _native.PmddTsp(c.shape[1], c.shape[0], c.ctypes.data_as(P32))
        lib = _native.gpu_lib()
        err = ctypes.create_string_buffer(512)
        self = cls.__new__(cls)
        self.dds = []
        self._lib = lib
        self.device = device
        self.count = n
        self.problem_type = 3
        self._h = lib.pmdd_resident_build_tsp(specs, n, device, err, len(err))
        if not self._h:
            raise CudaEnumerationError(1, err.value.decode(errors="replace"))
        return self

    @property
    def device_bytes(self) -> int:
        return self._lib.pmdd_resident_bytes(self._h)

    def dd_info(self, i: int) -> dict:
        shape = (ctypes.c_int32 * 5)()
        widths = (ctypes.c_int64 * 4)()
        if self._lib.pmdd_resident_dd_shape(self._h, i, shape, widths) != _native.PMDD_OK:
            raise IndexError(i)
        return {"nobjs": shape[0], "num_layers": shape[1], "num_nodes": shape[2], "num_arcs": shape[3],
                "num_weights": shape[4], "original_width": widths[0], "original_num_nodes": widths[1],
                "reduced_width": widths[2], "reduced_num_nodes": widths[3]}

    def dd_arrays(self, i: int) -> dict:
        """Host copy of DD i's flat arrays (same keys as DecisionDiagram.arrays)."""
        info = self.dd_info(i)
        d, L, N, A, K = (info[k] for k in ("nobjs", "num_layers", "num_nodes", "num_arcs", "num_weights"))
        out = {"layer_offsets": np.zeros(L + 1, np.int32), "in_arc_offsets": np.zeros(N + 1, np.int32),
               "arc_src": np.zeros(max(A, 1), np.int32), "arc_weight": np.zeros(max(A, 1), np.int32),
               "weights": np.zeros((K, d), np.int32), "min_weight": np.zeros(N, np.int32)}
        P32 = ctypes.POINTER(ctypes.c_int32)
        err = ctypes.create_string_buffer(512)
        rc = self._lib.pmdd_resident_dd_copy(self._h, i, *(out[k].ctypes.data_as(P32) for k in
                                                           ("layer_offsets", "in_arc_offsets", "arc_src",
                                                            "arc_weight", "weights", "min_weight")), err, len(err))
        if rc != _native.PMDD_OK:
            raise CudaEnumerationError(rc, err.value.decode(errors="replace"))
        out["arc_src"] = out["arc_src"][:A]
        out["arc_weight"] = out["arc_weight"][:A]
        return out

    def enumerate(self, method: int = 1, state_dominance: int = 0, max_cand: int = DEFAULT_MAX_CAND,
                  max_prod: int = DEFAULT_MAX_PROD, stats: Optional[dict] = None, keep: bool = True) -> list:
        n = self.count
        ptype = self.problem_type
        o = _options(method, ptype, state_dominance, True, max_cand, max_prod, self.device)
        outs = (_native.PmddFrontier * max(n, 1))()
        status = (ctypes.c_int32 * max(n, 1))()
        st = _native.PmddStats()
        err = ctypes.create_string_buffer(512)
        rc = self._lib.pmdd_resident_enumerate(self._h, ctypes.byref(o), outs, status, ctypes.byref(st), err,
                                               len(err))
        try:
            if rc != _native.PMDD_OK:
                raise CudaEnumerationError(rc, err.value.decode(errors="replace"))
            res = [_to_array(outs[i]) for i in range(n)] if keep else [int(outs[i].num_points) for i in range(n)]
        finally:
            for i in range(n):
                self._lib.pmdd_frontier_free(ctypes.byref(outs[i]))
        if stats is not None:
            stats.update(st.as_dict())
        return res

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pmdd_resident_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- the seam mirror
def topdown_cuda_enumerate(bdd: DecisionDiagram, maximization: bool = True, problem_type: int = 1,
                           state_dominance: int = 0, stats: Optional[dict] = None,
                           gpu_batch_size: int = DEFAULT_MAX_CAND) -> np.ndarray:
    """Method 1 on a BDD (reference: topdown_cuda_enumerate, src/pmdd/enum/gpu/enum.cu:55-63)."""
    return enumerate_dd(bdd, 1, problem_type, state_dominance, maximization, gpu_batch_size, DEFAULT_MAX_PROD,
                        stats=stats)


def topdown_mdd_cuda_enumerate(mdd: DecisionDiagram, stats: Optional[dict] = None,
                               gpu_batch_size: int = DEFAULT_MAX_CAND) -> np.ndarray:
    """Method 1 on an MDD (reference: topdown_mdd_cuda_enumerate, src/pmdd/enum/gpu/enum.cu:65-71)."""
    return enumerate_dd(mdd, 1, 3, 0, True, gpu_batch_size, DEFAULT_MAX_PROD, stats=stats)


def coupled_cuda_enumerate(mdd: DecisionDiagram, stats: Optional[dict] = None,
                           gpu_batch_size: int = DEFAULT_MAX_CAND,
                           gpu_max_prod: int = DEFAULT_MAX_PROD) -> np.ndarray:
    """Method 3 on an MDD (reference: coupled_cuda_enumerate, src/pmdd/enum/gpu/enum.cu:73-79)."""
    return enumerate_dd(mdd, 3, 3, 0, True, gpu_batch_size, gpu_max_prod, stats=stats)


def coupled_bdd_cuda_enumerate(bdd: DecisionDiagram, maximization: bool = True, problem_type: int = 1,
                               state_dominance: int = 0, stats: Optional[dict] = None,
                               gpu_batch_size: int = DEFAULT_MAX_CAND,
                               gpu_max_prod: int = DEFAULT_MAX_PROD) -> np.ndarray:
    """Method 3 on a BDD (reference: coupled_bdd_cuda_enumerate, src/pmdd/enum/gpu/enum.cu:595-756).
    Like the reference, the coupled path applies no state dominance."""
    return enumerate_dd(bdd, 3, problem_type, 0, maximization, gpu_batch_size, gpu_max_prod, stats=stats)
