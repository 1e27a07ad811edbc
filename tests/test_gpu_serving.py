"""The served request loop under continuous arrivals, a memory budget and failures.

* Every result of a mixed stream (knapsack and set packing by methods 1 and 3, TSP by
  methods 3 and 1) submitted a few at a time between engine steps, on a seeded
  schedule, equals the same request enumerated alone and, for the served list of the
  throughput run, the reference binary's frontier (tests/golden/headline/served.json).
* A small budget makes requests queue; a request that cannot fit finishes with
  PMDD_ERR_OOM while the others finish correctly (the reference's GPU path returns
  NULL and its CLI exits, src/pmdd/main.cpp:338-345).
* Cancelling a queued and a running request of the light lane, and a running one of the
  heavy lane, finishes them with PMDD_ERR_CANCELLED.
* Device allocations failed by the server's test hook fail requests with PMDD_ERR_OOM,
  never the server: every other result stays exact and later requests are served.
* The two lanes: small requests (DDs of at most 2^17 arcs) submitted beside a large one
  (a 4-objective knapsack n=60) finish before it, each equal to its lone frontier; a
  request run until nothing is pending is then polled, in either lane; with
  PMDD_SERVER_LANES=1 (one engine, in a child process) the same requests give the same
  frontiers.
"""
import json

import numpy as np
import pytest

import oracle
import pmdd_b200 as P
from conftest import frontier_digest, headline
from pmdd_b200 import instances

pytestmark = pytest.mark.gpu

OK, OOM, CANCELLED = 0, 3, 7


def _request(ptype, text, method, tag):
    """(kind, payload, method, lone DD): TSP requests go in by their cost matrices."""
    dd = P.DecisionDiagram.from_text(text, ptype, 3)
    if ptype == 3:
        return ("tsp", instances.tsp_arrays_from_tag(tag), method, dd)
    return ("dd", dd, method, dd)


def _submit(srv, req, rid):
    kind, payload, method, _ = req
    rc = srv.submit_tsp(payload, rid, method=method) if kind == "tsp" else srv.submit(payload, rid, method=method)
    assert rc == 0


def _drive(srv, reqs, rng, per_step=(0, 4)):
    """Submits reqs a random number at a time between single engine steps; returns
    {req_id: ServedResult}."""
    out = {}
    nxt = 0
    while len(out) < len(reqs):
        for _ in range(int(rng.integers(*per_step))):
            if nxt < len(reqs):
                _submit(srv, reqs[nxt], nxt)
                nxt += 1
        if srv.pending() == 0:
            if nxt < len(reqs):
                _submit(srv, reqs[nxt], nxt)
                nxt += 1
            continue
        srv.run(1)
        while True:
            r = srv.poll()
            if r is None:
                break
            out[r.req_id] = r
    return out


def test_served_mix_equals_alone_and_reference():
    mix = instances.served_mix(100, 50)
    ref = headline("served.json")["lists"]["50"]["results"]
    reqs = [_request(p, t, m, tag) for p, t, m, tag in mix]
    # the other method for a sample of each problem type (checked against lone runs and the oracle)
    extra = [(1, instances.knapsack_text(20 + 3 * i, 3, 900 + i), 3, f"kp3_m3_{i}") for i in range(4)] + \
            [(2, instances.setpacking_text(60 + 5 * i, 20, 3, 910 + i), 3, f"sp3_m3_{i}") for i in range(4)] + \
            [(3, instances.tsp_text(9 + i % 2, 3, 920 + i), 1, f"tsp3_n{9 + i % 2}_s{920 + i}") for i in range(4)]
    reqs += [_request(p, t, m, tag) for p, t, m, tag in extra]
    srv = P.Server(budget_bytes=1 << 30, max_slots=4)  # per lane: a queue forms
    try:
        got = _drive(srv, reqs, np.random.default_rng(7))
        info = srv.info()
    finally:
        srv.close()
    assert info["running_peak"] > 1 and info["queued_peak"] > 0
    assert info["completed"] == len(reqs) and info["failed"] == 0 and info["rejected"] == 0
    for i, (kind, payload, method, dd) in enumerate(reqs):
        r = got[i]
        assert r.status == OK, (i, r.error)
        alone = P.enumerate_dd(dd, method=method)
        assert frontier_digest(r.frontier) == frontier_digest(alone), i
        if i < len(ref):
            assert frontier_digest(r.frontier) == ref[i]["sha256"], mix[i][3]
        else:
            assert frontier_digest(r.frontier) == frontier_digest(oracle.enumerate(dd, method)), i


def test_budget_queues_requests_and_fails_only_the_one_that_cannot_fit():
    big = P.DecisionDiagram.from_text(instances.knapsack_text(60, 4, 0), 1, 4)  # ~120 MB of frontier slots
    small = [P.DecisionDiagram.from_text(instances.knapsack_text(34 + i % 7, 3, 700 + i), 1, 3) for i in range(16)]
    srv = P.Server(budget_bytes=64 << 20)
    try:
        assert srv.submit(big, 0, method=1) == 0
        for i, dd in enumerate(small):
            assert srv.submit(dd, 1 + i, method=1) == 0
        got = {}
        while srv.pending() > 0:
            srv.run(0)
            while (r := srv.poll()) is not None:
                got[r.req_id] = r
        info = srv.info()
    finally:
        srv.close()
    assert got[0].status == OOM and "memory" in got[0].error
    for i, dd in enumerate(small):
        r = got[1 + i]
        assert r.status == OK, r.error
        assert frontier_digest(r.frontier) == frontier_digest(oracle.enumerate(dd, 1))
    assert info["queued_peak"] > 0 and info["failed"] + info["rejected"] == 1
    assert info["peak_used_bytes"] <= info["budget_bytes"]


def test_cancel_queued_and_running_requests():
    # a, b, c: light lane (77011, 63097, 47735 arcs); d: heavy lane (673929 arcs, ~30 ms)
    a = P.DecisionDiagram.from_text(instances.setpacking_text(100, 20, 3, 3), 2, 3)
    b = P.DecisionDiagram.from_text(instances.knapsack_text(30, 3, 5), 1, 3)
    c = P.DecisionDiagram.from_text(instances.knapsack_text(28, 3, 6), 1, 3)
    d = P.DecisionDiagram.from_text(instances.knapsack_text(60, 4, 0), 1, 4)
    srv = P.Server(max_slots=2)
    try:
        for rid, dd in enumerate((a, b, c, d)):
            assert srv.submit(dd, rid, method=1) == 0
        srv.run(1)
        assert srv.info()["running"] >= 2 and srv.info()["queued"] >= 1
        assert srv.cancel(2) and srv.cancel(0) and srv.cancel(3)
        got = {}
        while srv.pending() > 0:
            srv.run(0)
            while (r := srv.poll()) is not None:
                got[r.req_id] = r
        while (r := srv.poll()) is not None:
            got[r.req_id] = r
        info = srv.info()
    finally:
        srv.close()
    assert got[0].status == CANCELLED and got[2].status == CANCELLED and got[3].status == CANCELLED
    assert got[1].status == OK
    assert frontier_digest(got[1].frontier) == frontier_digest(oracle.enumerate(b, 1))
    assert info["cancelled"] == 3


@pytest.mark.parametrize("count", [1, 20, 200])
def test_injected_allocation_failures_fail_requests_not_the_server(count):
    specs = [(1, instances.knapsack_text(24 + 2 * i, 3, 800 + i), 1, "") for i in range(3)] + \
            [(2, instances.setpacking_text(60, 20, 3, 810), 1, ""), (2, instances.setpacking_text(64, 20, 3, 811), 3, ""),
             (3, instances.tsp_text(9, 3, 812), 3, "tsp3_n9_s812")]
    reqs = [_request(*s) for s in specs]
    lone = [frontier_digest(P.enumerate_dd(r[3], method=r[2])) for r in reqs]
    outcomes = []
    for after in (0, 2, 5, 9, 14, 22, 35):
        srv = P.Server(budget_bytes=256 << 20)
        try:
            for i, r in enumerate(reqs):
                _submit(srv, r, i)
            srv.run(1)
            srv.inject_alloc_failures(after, count)
            got = {}
            while srv.pending() > 0:
                assert srv.run(0) >= 0
                while (x := srv.poll()) is not None:
                    got[x.req_id] = x
            for i in range(len(reqs)):
                assert got[i].status in (OK, OOM), (after, i, got[i].status, got[i].error)
                if got[i].status == OK:
                    assert frontier_digest(got[i].frontier) == lone[i], (after, i)
                else:
                    assert "memory" in got[i].error
                outcomes.append(got[i].status)
            # the server keeps serving once the failures have passed
            srv.inject_alloc_failures(0, 0)
            _submit(srv, reqs[0], 99)
            while srv.pending() > 0:
                srv.run(0)
            x = srv.poll()
            assert x.req_id == 99 and x.status == OK and frontier_digest(x.frontier) == lone[0]
            assert srv.info()["injected_alloc_failures"] > 0
        finally:
            srv.close()
    assert OK in outcomes
    if count >= 20:
        assert OOM in outcomes


LANE_CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
sys.path.insert(0, {tests!r})
import pmdd_b200 as P
from conftest import frontier_digest
from test_gpu_serving import _lane_requests, _drive_all
srv = P.Server()
out = _drive_all(srv, _lane_requests())
srv.close()
print(json.dumps({{str(k): frontier_digest(r.frontier) for k, r in out.items()}}))
"""


def _lane_requests():
    """A large request first (4-objective knapsack n=60, heavy lane), then small ones
    (TSP 9 cities by method 3, knapsack n=30 and set packing n=70: light lane)."""
    big = P.DecisionDiagram.from_text(instances.knapsack_text(60, 4, 0), 1, 4)
    small = [_request(3, instances.tsp_text(9, 3, 930 + i), 3, f"tsp3_n9_s{930 + i}") for i in range(4)] + \
            [_request(1, instances.knapsack_text(30, 3, 940 + i), 1, "") for i in range(3)] + \
            [_request(2, instances.setpacking_text(70, 20, 3, 950 + i), 1, "") for i in range(3)]
    return [("dd", big, 1, big)] + small


def _drive_all(srv, reqs):
    for i, r in enumerate(reqs):
        _submit(srv, r, i)
    out = {}
    while len(out) < len(reqs):
        assert srv.run(0) >= 0
        while (x := srv.poll()) is not None:
            out[x.req_id] = x
    return out


def test_small_requests_pass_a_large_one():
    import subprocess
    import sys

    from conftest import ROOT

    reqs = _lane_requests()
    srv = P.Server()
    try:
        got = _drive_all(srv, reqs)
    finally:
        srv.close()
    for i, (kind, payload, method, dd) in enumerate(reqs):
        assert got[i].status == OK, (i, got[i].error)
        assert frontier_digest(got[i].frontier) == frontier_digest(P.enumerate_dd(dd, method=method)), i
    # every small request finished before the large one that was submitted first
    assert max(got[i].finish_s for i in range(1, len(reqs))) < got[0].finish_s
    # run until nothing is pending, then poll: a heavy-lane result is pending until a run
    # call has reported it (bounded loop: a regression must fail, not hang)
    srv = P.Server()
    try:
        for i in (0, 1):
            _submit(srv, reqs[i], 100 + i)
            for _ in range(200000):
                if srv.pending() == 0:
                    break
                srv.run(0)
            assert srv.pending() == 0
            x = srv.poll()
            assert x is not None and x.req_id == 100 + i and x.status == OK
            assert frontier_digest(x.frontier) == frontier_digest(got[i].frontier)
    finally:
        srv.close()
    env = dict(__import__("os").environ, PMDD_SERVER_LANES="1")
    p = subprocess.run([sys.executable, "-c", LANE_CHILD.format(root=ROOT, tests=__import__("os").path.join(ROOT, "tests"))],
                       env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    one = json.loads(p.stdout.strip().splitlines()[-1])
    assert one == {str(i): frontier_digest(got[i].frontier) for i in range(len(reqs))}


def test_prepared_tsp_structures():
    """pmdd_server_prepare_tsp builds a size's structure in both lanes up front; requests of
    that size then give their lone frontiers, and sizes outside 2..20 cities are refused."""
    srv = P.Server()
    try:
        for n in (9, 11):
            srv.prepare_tsp(n)
        with pytest.raises(Exception):
            srv.prepare_tsp(40)
        reqs = [_request(3, instances.tsp_text(n, 3, 960 + n), m, f"tsp3_n{n}_s{960 + n}") for n in (9, 11) for m in (1, 3)]
        got = _drive_all(srv, reqs)
    finally:
        srv.close()
    for i, (kind, payload, method, dd) in enumerate(reqs):
        assert got[i].status == OK, got[i].error
        assert frontier_digest(got[i].frontier) == frontier_digest(P.enumerate_dd(dd, method=method)), i
