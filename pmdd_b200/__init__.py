"""pmdd_b200: B200-native exact Pareto-frontier enumeration over decision diagrams.

The hot path (per-layer arc expansion, dominance filtering, method-3 cutset
coupling) runs in hand-written sm_100a CUDA (libpmdd_gpu.so); instance parsing and
DD construction run in C++ (libpmdd_host.so).  See include/pmdd.h for the C ABI.
"""
from .dd import (PROBLEM_KNAPSACK, PROBLEM_SETPACKING, PROBLEM_TSP, DDBuildError, DecisionDiagram,
                 sort_lexicographic_ascending)
from .enumerate import (DEFAULT_MAX_CAND, DEFAULT_MAX_PROD, CudaEnumerationError, ResidentSet, pareto_filter,
                        coupled_bdd_cuda_enumerate,
                        coupled_cuda_enumerate, enumerate_batch, enumerate_dd, topdown_cuda_enumerate,
                        topdown_mdd_cuda_enumerate)
from .server import Server

__all__ = [
    "PROBLEM_KNAPSACK", "PROBLEM_SETPACKING", "PROBLEM_TSP", "DDBuildError", "DecisionDiagram",
    "sort_lexicographic_ascending", "ResidentSet", "pareto_filter", "DEFAULT_MAX_CAND", "DEFAULT_MAX_PROD", "CudaEnumerationError",
    "coupled_bdd_cuda_enumerate", "coupled_cuda_enumerate", "enumerate_batch", "enumerate_dd",
    "topdown_cuda_enumerate", "topdown_mdd_cuda_enumerate", "Server",
]
