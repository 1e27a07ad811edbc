"""ctypes view of the two in-tree native libraries.

libpmdd_host.so  -- instance parsers and exact DD constructors (include/pmdd_host.h)
libpmdd_gpu.so   -- the sm_100a enumeration engine (include/pmdd.h)

The GPU library is loaded on first use and its absence is an error: there is no CPU
fallback behind the enumeration entry points.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "lib")
BIN_DIR = os.path.join(_HERE, "bin")

c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
P_i32 = ctypes.POINTER(ctypes.c_int32)


class PmddDD(ctypes.Structure):
    _fields_ = [
        ("nobjs", c_i32),
        ("num_layers", c_i32),
        ("num_nodes", c_i32),
        ("num_arcs", c_i32),
        ("num_weights", c_i32),
        ("layer_offsets", P_i32),
        ("in_arc_offsets", P_i32),
        ("arc_src", P_i32),
        ("arc_weight", P_i32),
        ("weights", P_i32),
        ("min_weight", P_i32),
        ("node_state", ctypes.POINTER(ctypes.c_uint64)),
        ("state_words", c_i32),
        ("reserved", c_i32),
    ]


class PmddKnapsack(ctypes.Structure):
    _fields_ = [
        ("n", c_i32),
        ("nobjs", c_i32),
        ("profits", P_i32),
        ("weights", P_i32),
        ("capacity", c_i32),
        ("reserved", c_i32),
    ]


class PmddTsp(ctypes.Structure):
    _fields_ = [
        ("n", c_i32),
        ("nobjs", c_i32),
        ("cost", P_i32),
    ]


class PmddOptions(ctypes.Structure):
    _fields_ = [
        ("method", c_i32),
        ("problem_type", c_i32),
        ("state_dominance", c_i32),
        ("maximization", c_i32),
        ("max_cand", c_i64),
        ("max_prod", c_i64),
        ("device", c_i32),
        ("reserved", c_i32),
    ]


class PmddFrontier(ctypes.Structure):
    _fields_ = [
        ("nobjs", c_i32),
        ("elem_bytes", c_i32),
        ("num_points", c_i64),
        ("points", ctypes.c_void_p),
    ]


class PmddStats(ctypes.Structure):
    _fields_ = [
        ("wall_pack_transfer_s", ctypes.c_double),
        ("wall_join_s", ctypes.c_double),
        ("kernel_expand_td_s", ctypes.c_double),
        ("kernel_dominance_s", ctypes.c_double),
        ("kernel_total_s", ctypes.c_double),
        ("gpu_mem_peak_used_bytes", c_i64),
        ("gpu_mem_peak_reserved_bytes", c_i64),
        ("work_candidates_total", c_i64),
        ("work_candidates_peak", c_i64),
        ("work_frontier_survivors_total", c_i64),
        ("work_frontier_peak_points", c_i64),
        ("work_join_products_total", c_i64),
        ("dominance_filtered_total", c_i64),
        ("layer_coupling", c_i32),
        ("layers_td", c_i32),
        ("layers_bu", c_i32),
        ("cutset_size", c_i32),
        ("gpu_launches", c_i64),
        ("device_elapsed_s", ctypes.c_double),
        ("work_tile_candidates_total", c_i64),
        ("work_tile_survivors_total", c_i64),
        ("tile_launches", c_i64),
        ("work_stair_candidates_total", c_i64),
        ("work_chained_layers", c_i64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PmddServerInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("submitted", "admitted", "completed", "failed", "rejected",
                                              "cancelled")] + \
               [(n, ctypes.c_int32) for n in ("queued", "running", "queued_peak", "running_peak")] + \
               [(n, ctypes.c_int64) for n in ("budget_bytes", "used_bytes", "peak_used_bytes",
                                              "reserved_growth_bytes", "injected_alloc_failures")]


class PmddResult(ctypes.Structure):
    _fields_ = [
        ("req_id", ctypes.c_uint64),
        ("status", c_i32),
        ("reserved", c_i32),
        ("frontier", PmddFrontier),
        ("submit_s", ctypes.c_double),
        ("admit_s", ctypes.c_double),
        ("finish_s", ctypes.c_double),
        ("error", ctypes.c_char * 160),
    ]


class PmddDDInfo(ctypes.Structure):
    _fields_ = [
        ("original_width", c_i64),
        ("reduced_width", c_i64),
        ("original_num_nodes", c_i64),
        ("reduced_num_nodes", c_i64),
        ("max_num_in_arcs", c_i64),
        ("total_num_in_arcs", c_i64),
        ("num_layers", c_i32),
        ("problem_type", c_i32),
    ]


# status codes (include/pmdd.h)
PMDD_OK = 0
STATUS_NAMES = {
    0: "OK",
    1: "INVALID",
    2: "CUDA",
    3: "OOM",
    4: "CAND_OVERFLOW",
    5: "TIMEOUT",
    6: "INTERNAL",
    7: "CANCELLED",
    8: "NO_DEVICE",
    9: "RANGE",
    10: "IO",
}

HOST_SYMBOLS = {
    "pmdd_build_from_file": (ctypes.c_void_p, [ctypes.c_char_p, c_i32, c_i32, ctypes.c_char_p, ctypes.c_size_t]),
    "pmdd_build_from_text": (ctypes.c_void_p, [ctypes.c_char_p, c_i32, c_i32, ctypes.c_char_p, ctypes.c_size_t]),
    "pmdd_host_dd_view": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PmddDD)]),
    "pmdd_host_dd_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PmddDDInfo)]),
    "pmdd_host_dd_layer_sizes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(c_i64), c_i32]),
    "pmdd_host_dd_free": (None, [ctypes.c_void_p]),
    "pmdd_sort_points_lex_ascending": (None, [P_i32, c_i64, c_i32]),
    "pmdd_write_frontier_csv_gz": (ctypes.c_int, [ctypes.c_void_p, c_i64, c_i32, c_i32, c_i32, ctypes.c_char_p,
                                                  ctypes.c_char_p, ctypes.c_size_t]),
    "pmdd_writer_create": (ctypes.c_void_p, [c_i32, ctypes.c_char_p, ctypes.c_size_t]),
    "pmdd_writer_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, c_i64, c_i32, c_i32, ctypes.c_char_p,
                                          ctypes.c_char_p, ctypes.c_char_p]),
    "pmdd_writer_pending": (c_i64, [ctypes.c_void_p]),
    "pmdd_writer_flush": (c_i64, [ctypes.c_void_p, ctypes.POINTER(c_i64), ctypes.c_char_p, ctypes.c_size_t]),
    "pmdd_writer_destroy": (None, [ctypes.c_void_p]),
}

GPU_SYMBOLS = {
    "pmdd_options_default": (None, [ctypes.POINTER(PmddOptions)]),
    "pmdd_frontier_free": (None, [ctypes.POINTER(PmddFrontier)]),
    "pmdd_enumerate": (
        ctypes.c_int,
        [ctypes.POINTER(PmddDD), ctypes.POINTER(PmddOptions), ctypes.POINTER(PmddFrontier),
         ctypes.POINTER(PmddStats), ctypes.c_char_p, ctypes.c_size_t],
    ),
    "pmdd_enumerate_batch": (
        ctypes.c_int,
        [ctypes.POINTER(PmddDD), c_i32, ctypes.POINTER(PmddOptions), ctypes.POINTER(PmddFrontier),
         P_i32, ctypes.POINTER(PmddStats), ctypes.c_char_p, ctypes.c_size_t],
    ),
    "pmdd_pareto_filter": (ctypes.c_int, [P_i32, c_i64, c_i32, P_i32, ctypes.POINTER(c_i64), c_i32, ctypes.c_char_p,
                                          ctypes.c_size_t]),
    "pmdd_pareto_filter_noalloc": (ctypes.c_int, [ctypes.c_void_p, c_i64, c_i32, ctypes.c_void_p,
                                                  ctypes.POINTER(c_i64), ctypes.c_void_p, ctypes.c_char_p,
                                                  ctypes.c_size_t]),
    "pmdd_resident_upload": (ctypes.c_void_p, [ctypes.POINTER(PmddDD), c_i32, c_i32, ctypes.c_char_p,
                                                ctypes.c_size_t]),
    "pmdd_resident_enumerate": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.POINTER(PmddOptions), ctypes.POINTER(PmddFrontier), P_i32,
         ctypes.POINTER(PmddStats), ctypes.c_char_p, ctypes.c_size_t],
    ),
    "pmdd_resident_bytes": (c_i64, [ctypes.c_void_p]),
    "pmdd_resident_build_knapsack": (ctypes.c_void_p, [ctypes.POINTER(PmddKnapsack), c_i32, c_i32, ctypes.c_char_p,
                                                       ctypes.c_size_t]),
    "pmdd_resident_build_tsp": (ctypes.c_void_p, [ctypes.POINTER(PmddTsp), c_i32, c_i32, ctypes.c_char_p,
                                                  ctypes.c_size_t]),
    "pmdd_server_submit_tsp": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PmddTsp), ctypes.POINTER(PmddOptions),
                                              ctypes.c_uint64]),
    "pmdd_server_prepare_tsp": (ctypes.c_int, [ctypes.c_void_p, c_i32]),
    "pmdd_resident_dd_shape": (ctypes.c_int, [ctypes.c_void_p, c_i32, P_i32, ctypes.POINTER(c_i64)]),
    "pmdd_resident_dd_copy": (ctypes.c_int, [ctypes.c_void_p, c_i32, P_i32, P_i32, P_i32, P_i32, P_i32, P_i32,
                                             ctypes.c_char_p, ctypes.c_size_t]),
    "pmdd_resident_free": (None, [ctypes.c_void_p]),
    "pmdd_server_create": (ctypes.c_void_p, [c_i32, c_i64, c_i32, ctypes.c_char_p, ctypes.c_size_t]),
    "pmdd_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PmddDD), ctypes.POINTER(PmddOptions),
                                          ctypes.c_uint64]),
    "pmdd_server_run": (ctypes.c_int, [ctypes.c_void_p, c_i32]),
    "pmdd_server_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PmddResult)]),
    "pmdd_server_cancel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "pmdd_server_pending": (ctypes.c_int, [ctypes.c_void_p]),
    "pmdd_server_destroy": (None, [ctypes.c_void_p]),
    "pmdd_server_get_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PmddServerInfo)]),
    "pmdd_server_inject_alloc_failures": (ctypes.c_int, [ctypes.c_void_p, c_i64, c_i64]),
    "pmdd_version": (ctypes.c_char_p, []),
    "pmdd_launch_count": (c_i64, []),
    "pmdd_tuned_mark_min": (c_i64, [ctypes.c_char_p, c_i32, c_i32]),
    "pmdd_tuned_lex_pair_max": (c_i64, [ctypes.c_char_p, c_i32, c_i32]),
    "pmdd_tuned_tile_window_max": (c_i64, [ctypes.c_char_p, c_i32, c_i32]),
}

_host = None
_gpu = None


def _bind(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def host_lib():
    """libpmdd_host.so (CPU-only; safe to load without a GPU)."""
    global _host
    if _host is None:
        path = os.path.join(LIB_DIR, "libpmdd_host.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run `make -C pmdd_b200` (or __graft_entry__.build())")
        _host = _bind(ctypes.CDLL(path), HOST_SYMBOLS)
    return _host


def gpu_lib():
    """libpmdd_gpu.so.  Raises if the library was not built: the enumeration path
    has no fallback."""
    global _gpu
    if _gpu is None:
        path = os.path.join(LIB_DIR, "libpmdd_gpu.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: the CUDA engine was not built (make -C pmdd_b200 gpu)")
        _gpu = _bind(ctypes.CDLL(path), GPU_SYMBOLS)
    return _gpu
