"""Several GPUs: replicas, no collective on the data path.

Enumeration requests are independent, so each GPU runs its own engine on its own
requests and nothing crosses between GPUs (the reference runs one request at a time on
device 0, src/pmdd/enum/gpu/enum.cu:46).  Two ways to use several GPUs:

* one process per GPU (torchrun): each rank takes its own slice of the request stream
  (`rank_stream`) and the ranks meet only for barriers and the max-over-ranks timing
  reduction (`max_over_ranks`);
* one process driving every GPU: `ReplicaServers` keeps one serving loop per device and a
  `Dispatcher` sends each request to the device with the most free memory budget.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional, Sequence

from . import instances


def rank_stream(rank: int, num_knapsack: int = 512, num_setpacking: int = 256, nobjs: int = 3):
    """The batched-stream workload of one rank: the same generator, seeds offset by the
    rank, so ranks never solve the same instance (weak scaling)."""
    per_rank = num_knapsack + num_setpacking
    return instances.stream_mix(num_knapsack, num_setpacking, nobjs, seed0=rank * per_rank)


def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """Largest value of x over all ranks (the job time of a timed region); x itself
    without a process group.  `device` is where the reduction tensor lives: "cpu" for
    gloo, a CUDA device for NCCL."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dd_budget_bytes(dd) -> int:
    """Device bytes a request is charged against its replica's budget: its DD arrays
    (int32) plus the bottom-up CSR, twice over for the frontiers in flight."""
    v = dd.view
    words = (v.num_layers + 1) + 2 * (v.num_nodes + 1) + 4 * v.num_arcs + v.num_weights * v.nobjs
    return 2 * 4 * int(words)


class Dispatcher:
    """Sends each request to the replica with the most free budget (budget minus the
    bytes of its requests in flight); ties go to the lowest index."""

    def __init__(self, budgets: Sequence[int]):
        if not budgets:
            raise ValueError("at least one replica")
        self.budgets = [int(b) for b in budgets]
        self.in_flight = [0] * len(self.budgets)
        self._owner: Dict[int, tuple] = {}

    def assign(self, req_id: int, cost: int) -> int:
        free = [b - f for b, f in zip(self.budgets, self.in_flight)]
        k = max(range(len(free)), key=lambda i: (free[i], -i))
        self.in_flight[k] += int(cost)
        self._owner[req_id] = (k, int(cost))
        return k

    def done(self, req_id: int) -> int:
        k, cost = self._owner.pop(req_id)
        self.in_flight[k] -= cost
        return k

    def pending(self) -> int:
        return len(self._owner)


class ReplicaServers:
    """One serving loop per device in this process; `submit` dispatches by free budget,
    `run` advances every replica, `poll` returns finished requests from any of them.
    `make_server(device)` builds a replica (pmdd_b200.Server by default)."""

    def __init__(self, devices: Sequence[int], budget_bytes: Optional[Sequence[int]] = None,
                 make_server: Optional[Callable[[int], object]] = None):
        if make_server is None:
            from .server import Server

            def make_server(dev):
                return Server(device=dev)
        self.devices = list(devices)
        self.servers = [make_server(d) for d in self.devices]
        budgets = list(budget_bytes) if budget_bytes is not None else [1 << 40] * len(self.devices)
        self.dispatcher = Dispatcher(budgets)

    def submit(self, dd, req_id: int, **kw) -> int:
        k = self.dispatcher.assign(req_id, dd_budget_bytes(dd))
        self.servers[k].submit(dd, req_id, **kw)
        return self.devices[k]

    def run(self, max_steps: int = 1) -> int:
        return sum(s.run(max_steps) for s in self.servers)

    def poll(self) -> List[object]:
        out = []
        for s in self.servers:
            while True:
                r = s.poll()
                if r is None:
                    break
                self.dispatcher.done(r.req_id)
                out.append(r)
        return out

    def pending(self) -> int:
        return self.dispatcher.pending()

    def close(self):
        for s in self.servers:
            close = getattr(s, "close", None)
            if close:
                close()
