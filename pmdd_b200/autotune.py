"""Autotuner for the filter crossovers, cached per (objectives, problem type).

Destinations too large for a shared-memory tile are filtered one of two ways: one
sort-filter-skyline block each (one SM per destination) or the GPU-wide pass that drops
what the largest-sum pivots dominate and sweeps the rest pairwise (every SM).  The size
from which the GPU-wide pass pays depends on the instance family.  For each requested
(objectives, problem type) this tuner times a calibration instance of that family under a
list of crossover sizes, each in a fresh process (the engine reads PMDD_BIG_MARK_MIN at
start-up), and under the engine's built-in behaviour (1025: every destination with more
candidates than a tile holds takes the GPU-wide pass), keeps the fastest, and writes the
choice to the tuning file the engine reads at start-up:

    {"version": 1, "entries": {"d<objectives>_p<problem type>": {"big_mark_min": n,
                                "seconds": {"<n>": device seconds, ...}, "instance": "..."}}}

A family for which the built-in behaviour is as fast as the best size gets an entry
without "big_mark_min" ({"builtin": true, ...}), which the engine reads as untuned.

Three-objective families also get "lex_pair_max": in the lexicographic tiles,
destinations of at most that many candidates are checked pairwise against the points
before them and larger ones by a staircase warp.  It is timed over PAIR_MAX_SIZES with the
chosen oversized crossover in place (PMDD_LEX_PAIR_MAX in a fresh process); sizes within
2 % of the fastest tie and the default (48) wins a tie, else the smallest.

Every family also gets "tile_window_max", the largest tile window (the candidates a tile's
destinations start within; a step's window is its candidates over six tiles per SM,
between 128 and this): timed over WINDOW_SIZES with the choices above in place
(PMDD_TILE_WINDOW_MAX in a fresh process); ties as for the pairwise limit, the default
(1024) winning, else the largest.

    python -m pmdd_b200.autotune --nobjs 3 5 --ptype 1 3 [--out PATH]

The file is PMDD_TUNING_FILE if set, else $XDG_CACHE_HOME/pmdd_b200/tuning.json or
~/.cache/pmdd_b200/tuning.json.  Without a file the engine uses 1025 for every family.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
from typing import Callable, Dict, Iterable, Optional, Sequence

from . import instances

CANDIDATE_SIZES = (1025, 4096, 16384, 65536, 1 << 40)
DEFAULT_MARK_MIN = 1025
PAIR_MAX_SIZES = (0, 16, 32, 48, 96, 256, 1024)
DEFAULT_PAIR_MAX = 48
WINDOW_SIZES = (256, 512, 1024)
DEFAULT_WINDOW = 1024


def tuning_path() -> str:
    p = os.environ.get("PMDD_TUNING_FILE")
    if p:
        return p
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "pmdd_b200", "tuning.json")


def calibration_instance(nobjs: int, problem_type: int):
    """(description, text) of the instance a family is tuned on: large enough that
    some destinations leave the tiles, small enough to run in seconds."""
    if problem_type == 1:
        n = {1: 120, 2: 90, 3: 60, 4: 50}.get(nobjs, 30)
        return f"knapsack n={n} seed 0", instances.knapsack_text(n, nobjs, 0)
    if problem_type == 2:
        return "set packing n=100 m=20 seed 0", instances.setpacking_text(100, 20, nobjs, 0)
    n = {1: 14, 2: 14, 3: 13, 4: 12}.get(nobjs, 11)
    return f"tsp n={n} seed 0", instances.tsp_text(n, nobjs, 0)


_CHILD = r"""
import json, sys
sys.path.insert(0, {root!r})
import pmdd_b200 as P
dd = P.DecisionDiagram.from_text(open({path!r}).read(), {ptype}, {nobjs})
best = None
for _ in range({repeats}):
    st = {{}}
    P.enumerate_dd(dd, method={method}, stats=st)
    best = st["device_elapsed_s"] if best is None else min(best, st["device_elapsed_s"])
print(json.dumps({{"seconds": best}}))
"""


def time_in_child(path: str, nobjs: int, problem_type: int, method: int, mark_min: Optional[int],
                  repeats: int = 3, timeout: float = 600.0, pair_max: Optional[int] = None,
                  window: Optional[int] = None) -> Optional[float]:
    """Best device time of `repeats` enumerations in a fresh process with the given
    oversized crossover (None: the engine's built-in behaviour, no tuning file),
    three-objective pairwise limit (None: the built-in 48) and largest tile window (None:
    the built-in 1024); None if the run fails or times out."""
    root = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
    code = _CHILD.format(root=root, path=path, ptype=problem_type, nobjs=nobjs, method=method, repeats=repeats)
    env = dict(os.environ, PMDD_TUNING_FILE=path + ".no-tuning.json")
    if mark_min is None:
        env.pop("PMDD_BIG_MARK_MIN", None)
    else:
        env["PMDD_BIG_MARK_MIN"] = str(int(mark_min))
    if pair_max is None:
        env.pop("PMDD_LEX_PAIR_MAX", None)
    else:
        env["PMDD_LEX_PAIR_MAX"] = str(int(pair_max))
    if window is None:
        env.pop("PMDD_TILE_WINDOW_MAX", None)
    else:
        env["PMDD_TILE_WINDOW_MAX"] = str(int(window))
    try:
        p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return None
    if p.returncode != 0:
        return None
    try:
        return float(json.loads(p.stdout.strip().splitlines()[-1])["seconds"])
    except (ValueError, KeyError, IndexError):
        return None


def choose(times: Dict[int, Optional[float]], builtin: Optional[float] = None) -> Optional[int]:
    """Fastest crossover, or None when the built-in behaviour (timed as `builtin`) is
    within 2 % of the fastest.  Sizes within 2 % of the fastest tie: the default wins a tie
    (a calibration run whose destinations never reach the crossover says nothing about
    it), otherwise the larger size (fewer GPU-wide passes); no usable timing -> the
    default."""
    ok = {k: v for k, v in times.items() if v is not None}
    if not ok:
        return None if builtin is not None else DEFAULT_MARK_MIN
    best = min(ok.values())
    if builtin is not None and builtin <= best * 1.02:
        return None
    tied = [k for k, v in ok.items() if v <= best * 1.02]
    return DEFAULT_MARK_MIN if DEFAULT_MARK_MIN in tied else max(tied)


def choose_pair_max(times: Dict[int, Optional[float]]) -> int:
    """Fastest pairwise limit; sizes within 2 % of the fastest tie, the default wins a
    tie, else the smallest; no usable timing -> the default."""
    ok = {k: v for k, v in times.items() if v is not None}
    if not ok:
        return DEFAULT_PAIR_MAX
    best = min(ok.values())
    tied = [k for k, v in ok.items() if v <= best * 1.02]
    return DEFAULT_PAIR_MAX if DEFAULT_PAIR_MAX in tied else min(tied)


def choose_window(times: Dict[int, Optional[float]]) -> int:
    """Fastest largest tile window; sizes within 2 % of the fastest tie, the default wins
    a tie, else the largest; no usable timing -> the default."""
    ok = {k: v for k, v in times.items() if v is not None}
    if not ok:
        return DEFAULT_WINDOW
    best = min(ok.values())
    tied = [k for k, v in ok.items() if v <= best * 1.02]
    return DEFAULT_WINDOW if DEFAULT_WINDOW in tied else max(tied)


def tune(families: Iterable[tuple], sizes: Sequence[int] = CANDIDATE_SIZES, method: int = 1,
         timer: Optional[Callable[..., Optional[float]]] = None, workdir: Optional[str] = None) -> Dict[str, dict]:
    """Tunes every (nobjs, problem_type) of `families`; returns the entries to store."""
    import tempfile

    timer = timer or time_in_child
    workdir = workdir or tempfile.mkdtemp()
    out = {}
    for nobjs, ptype in families:
        desc, text = calibration_instance(nobjs, ptype)
        path = os.path.join(workdir, f"cal_d{nobjs}_p{ptype}.dat")
        with open(path, "w") as f:
            f.write(text)
        times = {int(s): timer(path, nobjs, ptype, method, int(s)) for s in sizes}
        builtin = timer(path, nobjs, ptype, method, None)
        seconds = {str(k): v for k, v in times.items()}
        seconds["builtin"] = builtin
        pick = choose(times, builtin)
        entry = {"builtin": True} if pick is None else {"big_mark_min": pick}
        pair = None
        if nobjs == 3:
            pt = {int(k): timer(path, nobjs, ptype, method, pick, pair_max=int(k)) for k in PAIR_MAX_SIZES}
            pair = entry["lex_pair_max"] = choose_pair_max(pt)
            entry["pair_max_seconds"] = {str(k): v for k, v in pt.items()}
        wt = {int(k): timer(path, nobjs, ptype, method, pick, pair_max=pair, window=int(k)) for k in WINDOW_SIZES}
        entry["tile_window_max"] = choose_window(wt)
        entry["window_seconds"] = {str(k): v for k, v in wt.items()}
        entry.update({"seconds": seconds, "instance": desc})
        out[f"d{nobjs}_p{ptype}"] = entry
    return out


def write(entries: Dict[str, dict], path: Optional[str] = None) -> str:
    """Merges `entries` into the tuning file (other families are kept)."""
    path = path or tuning_path()
    data = {"version": 1, "entries": {}}
    if os.path.exists(path):
        try:
            with open(path) as f:
                old = json.load(f)
            data["entries"].update(old.get("entries", {}))
        except (OSError, ValueError):
            pass
    data["entries"].update(entries)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1)
    os.replace(tmp, path)
    return path


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--nobjs", type=int, nargs="+", default=[3])
    ap.add_argument("--ptype", type=int, nargs="+", default=[1, 2, 3])
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    entries = tune([(d, p) for d in args.nobjs for p in args.ptype])
    path = write(entries, args.out)
    for k, v in entries.items():
        print(k, v.get("big_mark_min", "built-in"), v.get("lex_pair_max", "-"), v.get("tile_window_max"), v["seconds"])
    print("written", path)


if __name__ == "__main__":
    main()
