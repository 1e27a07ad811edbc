"""Decision diagrams built by the host front end (libpmdd_host.so).

`DecisionDiagram` owns one compiled flat DD (include/pmdd.h layout).  It plays the
role of the reference's BDD / MDD objects at the GPU seam: the problem-specific
constructors (knapsack BDD, set-packing independent-set BDD, TSP MDD) run in C++
and the result is handed to the engine without conversion.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native

PROBLEM_KNAPSACK = 1
PROBLEM_SETPACKING = 2
PROBLEM_TSP = 3


class DDBuildError(RuntimeError):
    pass


class DecisionDiagram:
    """An exact DD for one instance, compiled for `nobjs` objectives."""

    def __init__(self, handle: int, problem_type: int, nobjs: int):
        self._h = ctypes.c_void_p(handle)
        self.problem_type = problem_type
        self.nobjs = nobjs
        self._view = _native.PmddDD()
        _native.host_lib().pmdd_host_dd_view(self._h, ctypes.byref(self._view))

    # ------------------------------------------------------------ constructors
    @classmethod
    def from_text(cls, text: str, problem_type: int, nobjs: int) -> "DecisionDiagram":
        err = ctypes.create_string_buffer(512)
        h = _native.host_lib().pmdd_build_from_text(text.encode(), problem_type, nobjs, err, len(err))
        if not h:
            raise DDBuildError(err.value.decode(errors="replace"))
        return cls(h, problem_type, nobjs)

    @classmethod
    def from_file(cls, path: str, problem_type: int, nobjs: int) -> "DecisionDiagram":
        err = ctypes.create_string_buffer(512)
        h = _native.host_lib().pmdd_build_from_file(str(path).encode(), problem_type, nobjs, err, len(err))
        if not h:
            raise DDBuildError(err.value.decode(errors="replace"))
        return cls(h, problem_type, nobjs)

    # ---------------------------------------------------------------- views
    @property
    def view(self) -> _native.PmddDD:
        """Borrowed pmdd_dd (valid while this object lives)."""
        return self._view

    @property
    def num_layers(self) -> int:
        return self._view.num_layers

    @property
    def num_nodes(self) -> int:
        return self._view.num_nodes

    @property
    def num_arcs(self) -> int:
        return self._view.num_arcs

    def info(self) -> dict:
        inf = _native.PmddDDInfo()
        _native.host_lib().pmdd_host_dd_info(self._h, ctypes.byref(inf))
        return {name: getattr(inf, name) for name, _ in inf._fields_}

    def layer_sizes(self) -> list:
        buf = (ctypes.c_int64 * self.num_layers)()
        _native.host_lib().pmdd_host_dd_layer_sizes(self._h, buf, self.num_layers)
        return list(buf)

    def arrays(self) -> dict:
        """Copies of the flat arrays (for tests and debugging)."""
        v = self._view

        def arr(ptr, n):
            if n == 0 or not ptr:
                return np.zeros(0, dtype=np.int32)
            return np.ctypeslib.as_array(ptr, shape=(n,)).copy()

        return {
            "layer_offsets": arr(v.layer_offsets, v.num_layers + 1),
            "in_arc_offsets": arr(v.in_arc_offsets, v.num_nodes + 1),
            "arc_src": arr(v.arc_src, v.num_arcs),
            "arc_weight": arr(v.arc_weight, v.num_arcs),
            "weights": arr(v.weights, v.num_weights * v.nobjs).reshape(v.num_weights, v.nobjs),
            "min_weight": arr(v.min_weight, v.num_nodes) if v.min_weight else None,
            "node_state": (np.ctypeslib.as_array(v.node_state, shape=(v.num_nodes, v.state_words)).copy()
                           if v.node_state and v.state_words > 0 else None),
        }

    def close(self):
        if self._h:
            _native.host_lib().pmdd_host_dd_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sort_lexicographic_ascending(points: np.ndarray) -> np.ndarray:
    """Ascending lexicographic order of a (F, d) int32 frontier (the reference's
    ParetoFrontier::sort_lexicographic_ascending)."""
    pts = np.ascontiguousarray(points, dtype=np.int32)
    if pts.shape[0] > 1:
        order = np.lexsort(pts.T[::-1])
        pts = pts[order]
    return pts
