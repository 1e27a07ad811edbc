"""Several GPUs = replicas (pmdd_b200/replicas.py): the host logic on CPU.

The ranks of `bench.py --gpus N` take disjoint slices of the request stream and meet
only in barriers and the max-over-ranks timing reduction; these run here as two gloo
ranks on 127.0.0.1.  The in-process dispatcher is driven with fake replicas.
"""
import os
import socket
from types import SimpleNamespace

import pytest
import torch.multiprocessing as mp

from pmdd_b200 import replicas


def test_rank_streams_are_disjoint():
    a = replicas.rank_stream(0, 16, 8)
    b = replicas.rank_stream(1, 16, 8)
    assert len(a) == len(b) == 24
    assert not ({t for _, _, t in a} & {t for _, _, t in b})
    assert replicas.rank_stream(0, 16, 8) == a  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t = replicas.max_over_ranks(1.5 + rank, dist, "cpu")
        tags = [tag for _, _, tag in replicas.rank_stream(rank, 8, 4)]
        everyone = [None] * world
        dist.all_gather_object(everyone, tags)
        dist.barrier()
        out[rank] = (t, everyone)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_and_streams():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for rank in range(world):
        t, everyone = res[rank]
        assert t == pytest.approx(2.5)  # max over ranks of 1.5 + rank
        assert not (set(everyone[0]) & set(everyone[1]))
    assert res[0][1] == res[1][1]


def test_max_over_ranks_without_a_group():
    assert replicas.max_over_ranks(3.25) == 3.25


def test_dispatcher_sends_to_the_freest_replica():
    d = replicas.Dispatcher([100, 300])
    assert d.assign(1, 150) == 1      # 100 vs 300 free
    assert d.assign(2, 10) == 1       # 100 vs 150
    assert d.assign(3, 50) == 1       # 100 vs 140
    assert d.assign(4, 10) == 0       # 100 vs 90
    assert d.done(1) == 1
    assert d.assign(5, 1) == 1        # 90 vs 240
    assert d.pending() == 4


class _FakeServer:
    def __init__(self, dev):
        self.dev, self.q, self.done = dev, [], []

    def submit(self, dd, req_id, **kw):
        self.q.append(req_id)

    def run(self, max_steps=1):
        n = len(self.q)
        self.done += [SimpleNamespace(req_id=r, status=0) for r in self.q]
        self.q = []
        return n

    def poll(self):
        return self.done.pop(0) if self.done else None


def _fake_dd(arcs):
    return SimpleNamespace(view=SimpleNamespace(num_layers=3, num_nodes=4, num_arcs=arcs, num_weights=2, nobjs=3))


def test_replica_servers_round_trip_with_fakes():
    rs = replicas.ReplicaServers([0, 1], budget_bytes=[10_000, 10_000], make_server=_FakeServer)
    devs = [rs.submit(_fake_dd(100 + i), i) for i in range(6)]
    assert set(devs) == {0, 1}        # both replicas get work
    assert rs.pending() == 6
    assert rs.run() == 6
    got = sorted(r.req_id for r in rs.poll())
    assert got == list(range(6)) and rs.pending() == 0
