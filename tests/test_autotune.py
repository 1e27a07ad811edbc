"""The autotuner (pmdd_b200/autotune.py) and the engine's reading of its tuning file
(pmdd_tuned_mark_min / _lex_pair_max / _tile_window_max, the same parser the engine uses
at start-up): the choices with a fake timer, and on the GPU that the engine applies a
tuned oversized crossover, pairwise limit and tile window."""
import json
import os

import pytest

from pmdd_b200 import _native, autotune


def test_choose_picks_fastest_and_breaks_ties_upward():
    assert autotune.choose({4096: 2.0, 65536: 1.0, 1 << 40: 1.5}) == 65536
    assert autotune.choose({4096: 1.00, 65536: 1.01, 262144: 3.0}) == 65536  # within 2 %: larger size
    assert autotune.choose({4096: None, 65536: None}) == autotune.DEFAULT_MARK_MIN
    assert autotune.choose({4096: None, 16384: 0.5}) == 16384
    flat = {1025: 0.0077, 4096: 0.0077, 16384: 0.0077, 1 << 40: 0.0077}  # crossover never reached
    assert autotune.choose(flat) == autotune.DEFAULT_MARK_MIN
    assert autotune.choose({16384: 1.0, 262144: 1.01, 1 << 40: 1.005}) == 1 << 40


def test_tune_with_a_fake_timer(tmp_path):
    calls = []

    def timer(path, nobjs, ptype, method, mark_min, pair_max=None, window=None):
        calls.append((nobjs, ptype, mark_min, pair_max, window))
        assert os.path.exists(path)
        if window is not None:  # with the other choices in place: 512 for d=3, a tie for d=5
            assert pair_max == (96 if nobjs == 3 else None)
            return 1.0 + (abs(window - 512) / 1e3 if nobjs == 3 else 0.0)
        if pair_max is not None:  # three objectives: the staircase pays from 96 candidates up
            assert nobjs == 3 and mark_min == 16384
            return 1.0 + abs(pair_max - 96) / 1e3
        if mark_min is None:  # the built-in behaviour: slower for d=3, fastest for d=5
            return 2.0 if nobjs == 3 else 0.5
        return 1.0 + abs(mark_min - 16384) / 1e6

    entries = autotune.tune([(3, 1), (5, 3)], sizes=(4096, 16384, 65536), timer=timer, workdir=str(tmp_path))
    assert set(entries) == {"d3_p1", "d5_p3"}
    assert entries["d3_p1"]["big_mark_min"] == 16384
    assert entries["d3_p1"]["lex_pair_max"] == 96
    assert entries["d5_p3"]["builtin"] is True and "big_mark_min" not in entries["d5_p3"]
    assert "lex_pair_max" not in entries["d5_p3"]
    assert entries["d3_p1"]["tile_window_max"] == 512
    assert entries["d5_p3"]["tile_window_max"] == autotune.DEFAULT_WINDOW
    assert len(calls) == 8 + len(autotune.PAIR_MAX_SIZES) + 2 * len(autotune.WINDOW_SIZES)
    # the engine reads a built-in entry as untuned, the other one as tuned
    path = autotune.write(entries, str(tmp_path / "t.json"))
    lib = _native.gpu_lib()
    assert lib.pmdd_tuned_mark_min(path.encode(), 3, 1) == 16384
    assert lib.pmdd_tuned_mark_min(path.encode(), 5, 3) == 0
    assert lib.pmdd_tuned_lex_pair_max(path.encode(), 3, 1) == 96
    assert lib.pmdd_tuned_lex_pair_max(path.encode(), 5, 3) == -1
    assert lib.pmdd_tuned_tile_window_max(path.encode(), 3, 1) == 512
    assert lib.pmdd_tuned_tile_window_max(path.encode(), 5, 3) == 1024
    assert lib.pmdd_tuned_tile_window_max(path.encode(), 4, 2) == -1


def test_choose_pair_max():
    assert autotune.choose_pair_max({0: 2.0, 48: 1.5, 96: 1.0}) == 96
    assert autotune.choose_pair_max({0: 1.0, 48: 1.01, 96: 1.3}) == 48  # within 2 %: the default
    assert autotune.choose_pair_max({0: 1.0, 16: 1.01, 48: 1.5}) == 0   # else the smallest
    assert autotune.choose_pair_max({0: None}) == autotune.DEFAULT_PAIR_MAX
    assert autotune.DEFAULT_PAIR_MAX in autotune.PAIR_MAX_SIZES


def test_default_is_among_the_timed_sizes():
    """A tie can only go to the default if the tuner times it; it is the engine's built-in
    crossover, one above the largest tile destination (kSmallMax + 1)."""
    assert autotune.DEFAULT_MARK_MIN in autotune.CANDIDATE_SIZES
    assert autotune.DEFAULT_MARK_MIN == 1025


def test_builtin_wins_ties():
    assert autotune.choose({4096: 1.0, 65536: 2.0}, builtin=1.01) is None
    assert autotune.choose({4096: 1.0, 65536: 2.0}, builtin=1.5) == 4096
    assert autotune.choose({4096: None}, builtin=1.0) is None


def test_calibration_instances_build():
    from pmdd_b200 import DecisionDiagram

    for nobjs, ptype in ((3, 1), (7, 1), (3, 2), (3, 3), (5, 3)):
        _, text = autotune.calibration_instance(nobjs, ptype)
        dd = DecisionDiagram.from_text(text, ptype, nobjs)
        assert dd.view.num_layers >= 2 and dd.view.nobjs == nobjs


def test_written_file_is_what_the_engine_reads(tmp_path):
    path = str(tmp_path / "tuning.json")
    autotune.write({"d3_p1": {"big_mark_min": 12345, "seconds": {}}, "d5_p3": {"big_mark_min": 777}}, path)
    autotune.write({"d4_p2": {"big_mark_min": 4242}}, path)  # merges, keeps the others
    data = json.load(open(path))
    assert set(data["entries"]) == {"d3_p1", "d5_p3", "d4_p2"}
    lib = _native.gpu_lib()
    assert lib.pmdd_tuned_mark_min(path.encode(), 3, 1) == 12345
    assert lib.pmdd_tuned_mark_min(path.encode(), 5, 3) == 777
    assert lib.pmdd_tuned_mark_min(path.encode(), 4, 2) == 4242
    assert lib.pmdd_tuned_mark_min(path.encode(), 3, 2) == 0
    assert lib.pmdd_tuned_mark_min(str(tmp_path / "missing.json").encode(), 3, 1) == 0


def test_tuning_path_follows_the_environment(monkeypatch, tmp_path):
    monkeypatch.setenv("PMDD_TUNING_FILE", str(tmp_path / "x.json"))
    assert autotune.tuning_path() == str(tmp_path / "x.json")
    monkeypatch.delenv("PMDD_TUNING_FILE")
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    assert autotune.tuning_path() == os.path.join(str(tmp_path), "pmdd_b200", "tuning.json")
    lib = _native.gpu_lib()
    autotune.write({"d2_p1": {"big_mark_min": 99}})
    assert lib.pmdd_tuned_mark_min(None, 2, 1) == 99


TUNED_CHILD = r"""
import sys, json
sys.path.insert(0, {root!r})
import numpy as np
import oracle
import pmdd_b200 as P
from pmdd_b200 import instances
dd = P.DecisionDiagram.from_text(instances.tsp_text(10, 5, 77), 3, 5)
st = {{}}
got = P.enumerate_dd(dd, method=1, stats=st)
ok = np.array_equal(oracle.sorted_set(np.asarray(got, dtype=np.int64)),
                    oracle.sorted_set(np.asarray(oracle.enumerate(dd, 1), dtype=np.int64)))
print(json.dumps({{"ok": bool(ok), "launches": st["gpu_launches"]}}))
"""


@pytest.mark.gpu
def test_engine_applies_the_tuned_crossover(tmp_path):
    """A tuning file that sends 5-objective TSP destinations of 1025+ candidates to the
    GPU-wide pass launches more kernels (plan, mark, write) than one that keeps them all on
    SFS blocks; the frontier is the same."""
    import subprocess
    import sys

    from conftest import ROOT

    def run(env_extra):
        env = dict(os.environ, **env_extra)
        env.pop("PMDD_BIG_MARK_MIN", None)
        p = subprocess.run([sys.executable, "-c", TUNED_CHILD.format(root=ROOT)], env=env, capture_output=True,
                           text=True, timeout=600)
        assert p.returncode == 0, p.stdout + p.stderr
        return json.loads(p.stdout.strip().splitlines()[-1])

    path = str(tmp_path / "tuning.json")
    autotune.write({"d5_p3": {"big_mark_min": 1025}}, path)
    never = str(tmp_path / "never.json")
    autotune.write({"d5_p3": {"big_mark_min": 1 << 40}}, never)
    tuned = run({"PMDD_TUNING_FILE": path})
    plain = run({"PMDD_TUNING_FILE": never})
    assert tuned["ok"] and plain["ok"]
    assert tuned["launches"] > plain["launches"]


LEX_CHILD = r"""
import sys, json
sys.path.insert(0, {root!r})
import numpy as np
import oracle
import pmdd_b200 as P
from pmdd_b200 import instances
dd = P.DecisionDiagram.from_text(instances.knapsack_text(40, 3, 0), 1, 3)
st = {{}}
got = P.enumerate_dd(dd, method=1, stats=st)
ok = np.array_equal(oracle.sorted_set(got), oracle.sorted_set(oracle.enumerate(dd, 1)))
print(json.dumps({{"ok": bool(ok), "stair": st["work_stair_candidates_total"],
                   "cand": st["work_candidates_total"]}}))
"""


@pytest.mark.gpu
def test_engine_applies_the_tuned_pair_max(tmp_path):
    """A tuning file whose three-objective knapsack entry sends every tile destination to
    the staircase warps (lex_pair_max 0) makes them filter far more candidates than one
    that keeps every tile destination pairwise (1024: only oversized destinations are
    left to staircases); the frontier is the same."""
    import subprocess
    import sys

    from conftest import ROOT

    def run(pair_max):
        path = str(tmp_path / f"t{pair_max}.json")
        autotune.write({"d3_p1": {"lex_pair_max": pair_max}}, path)
        env = dict(os.environ, PMDD_TUNING_FILE=path)
        env.pop("PMDD_LEX_PAIR_MAX", None)
        env.pop("PMDD_LEX_TILES", None)
        p = subprocess.run([sys.executable, "-c", LEX_CHILD.format(root=ROOT)], env=env, capture_output=True,
                           text=True, timeout=600)
        assert p.returncode == 0, p.stdout + p.stderr
        return json.loads(p.stdout.strip().splitlines()[-1])

    all_stair, all_pair = run(0), run(1024)
    assert all_stair["ok"] and all_pair["ok"]
    assert all_stair["stair"] > 0.9 * all_stair["cand"]
    assert all_pair["stair"] < 0.05 * all_pair["cand"]


def test_choose_window():
    assert autotune.choose_window({256: 1.0, 512: 2.0, 1024: 3.0}) == 256
    assert autotune.choose_window({256: 1.0, 512: 1.01, 1024: 1.015}) == autotune.DEFAULT_WINDOW
    assert autotune.choose_window({256: 1.0, 512: 1.01, 1024: 2.0}) == 512
    assert autotune.choose_window({256: None, 512: None}) == autotune.DEFAULT_WINDOW


WINDOW_CHILD = r"""
import sys, json
sys.path.insert(0, {root!r})
import numpy as np
import oracle
import pmdd_b200 as P
from pmdd_b200 import instances
from conftest import frontier_digest
dds = [P.DecisionDiagram.from_text(instances.knapsack_text(40, 3, s), 1, 3) for s in range(16)]
got = P.enumerate_batch(dds, method=1)
print(json.dumps({{"digests": [frontier_digest(g) for g in got]}}))
"""


@pytest.mark.gpu
def test_engine_applies_the_tuned_tile_window(tmp_path):
    """A tuning file that caps the three-objective knapsack family's tile window at 256
    makes the steps of a 16-instance batch (up to ~10^6 candidates, so a 1024 window
    otherwise) use several times more tiles (the PMDD_TRACE step lines' tiles= count) than
    one that leaves it at 1024; the frontiers are the same."""
    import re
    import subprocess
    import sys

    from conftest import ROOT

    def run(window):
        path = str(tmp_path / f"w{window}.json")
        autotune.write({"d3_p1": {"tile_window_max": window}}, path)
        env = dict(os.environ, PMDD_TUNING_FILE=path, PMDD_TRACE="1", PMDD_CHAIN_LAYERS="0")
        env.pop("PMDD_TILE_WINDOW_MAX", None)
        p = subprocess.run([sys.executable, "-c", WINDOW_CHILD.format(root=ROOT)], env=env, capture_output=True,
                           text=True, timeout=600, cwd=os.path.join(ROOT, "tests"))
        assert p.returncode == 0, p.stdout + p.stderr
        tiles = sum(int(t) for t in re.findall(r" tiles=(\d+)", p.stderr))
        return json.loads(p.stdout.strip().splitlines()[-1])["digests"], tiles

    d256, t256 = run(256)
    d1024, t1024 = run(1024)
    assert d256 == d1024
    assert t256 > 2 * t1024
