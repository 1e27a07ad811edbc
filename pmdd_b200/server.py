"""Served request loop over libpmdd_gpu.so's pmdd_server_* entry points.

Requests are admitted as slots and HBM budget free up; every admitted request
advances one DD layer per engine step (or several, when a small step chains layers),
sharing each launch with the others (continuous batching).  Small requests (DDs of at
most 2^17 arcs) run in a light lane on the device's highest-priority stream, which
run() steps in the calling thread; larger ones in a heavy lane that a worker thread of
the server steps, so the small ones do not wait for their steps.  A server is used from
one thread at a time.  Timestamps are host monotonic seconds.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _native
from .dd import DecisionDiagram
from .enumerate import DEFAULT_MAX_CAND, DEFAULT_MAX_PROD, CudaEnumerationError, _options, _to_array


@dataclass
class ServedResult:
    req_id: int
    status: int
    frontier: np.ndarray
    submit_s: float
    admit_s: float
    finish_s: float
    error: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def latency_s(self) -> float:
        return self.finish_s - self.submit_s


class Server:
    def __init__(self, device: int = 0, budget_bytes: int = 0, max_slots: int = 0):
        lib = _native.gpu_lib()
        err = ctypes.create_string_buffer(512)
        self._h = lib.pmdd_server_create(device, int(budget_bytes), int(max_slots), err, len(err))
        if not self._h:
            raise CudaEnumerationError(8, err.value.decode(errors="replace"))
        self._lib = lib
        self._keep = {}   # req_id -> DecisionDiagram kept alive until submitted (the server copies it)

    def submit(self, dd: DecisionDiagram, req_id: int, method: int = 1, state_dominance: int = 0,
               max_cand: int = DEFAULT_MAX_CAND, max_prod: int = DEFAULT_MAX_PROD) -> int:
        o = _options(method, dd.problem_type, state_dominance, True, max_cand, max_prod, 0)
        view = dd.view
        return self._lib.pmdd_server_submit(self._h, ctypes.byref(view), ctypes.byref(o), ctypes.c_uint64(req_id))

    def submit_tsp(self, cost, req_id: int, method: int = 3, max_cand: int = DEFAULT_MAX_CAND,
                   max_prod: int = DEFAULT_MAX_PROD) -> int:
        """A TSP request by its cost matrices (nobjs, n, n): the server's shared n-city
        structure is used and only the weight table is uploaded."""
        c = np.ascontiguousarray(cost, dtype=np.int32)
        if c.ndim != 3 or c.shape[1] != c.shape[2]:
            raise ValueError("costs must be (nobjs, n, n)")
        spec = _native.PmddTsp(c.shape[1], c.shape[0], c.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        o = _options(method, 3, 0, True, max_cand, max_prod, 0)
        return self._lib.pmdd_server_submit_tsp(self._h, ctypes.byref(spec), ctypes.byref(o), ctypes.c_uint64(req_id))

    def prepare_tsp(self, n: int) -> None:
        """Builds the shared n-city MDD structure now instead of at the first TSP request
        of that size."""
        rc = self._lib.pmdd_server_prepare_tsp(self._h, int(n))
        if rc != 0:
            raise CudaEnumerationError(rc, f"building the {n}-city structure failed")

    def run(self, max_steps: int = 0) -> int:
        r = self._lib.pmdd_server_run(self._h, max_steps)
        if r < 0:
            raise CudaEnumerationError(2, "engine step failed")
        return r

    def poll(self) -> Optional[ServedResult]:
        res = _native.PmddResult()
        if not self._lib.pmdd_server_poll(self._h, ctypes.byref(res)):
            return None
        try:
            pts = _to_array(res.frontier)
        finally:
            self._lib.pmdd_frontier_free(ctypes.byref(res.frontier))
        return ServedResult(int(res.req_id), int(res.status), pts, res.submit_s, res.admit_s, res.finish_s,
                            res.error.decode(errors="replace"))

    def cancel(self, req_id: int) -> bool:
        return self._lib.pmdd_server_cancel(self._h, ctypes.c_uint64(req_id)) == 0

    def pending(self) -> int:
        return self._lib.pmdd_server_pending(self._h)

    def info(self) -> dict:
        """Serving counters and memory figures (pmdd_server_info)."""
        inf = _native.PmddServerInfo()
        self._lib.pmdd_server_get_info(self._h, ctypes.byref(inf))
        return {name: getattr(inf, name) for name, _ in inf._fields_}

    def inject_alloc_failures(self, after: int, count: int) -> None:
        """Test hook: after `after` more device allocations, the next `count` fail."""
        if self._lib.pmdd_server_inject_alloc_failures(self._h, int(after), int(count)) != 0:
            raise ValueError("after and count must be >= 0")

    def close(self):
        if self._h:
            self._lib.pmdd_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
