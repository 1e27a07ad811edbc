"""Frontier CSV.gz / stats JSONL writers (libpmdd_host.so, pmdd_b200.writer): the
decompressed CSV equals the reference's output byte for byte, and the asynchronous
writer loses, tears or reorders nothing within a file."""
import gzip
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import golden_cases
from pmdd_b200 import DecisionDiagram
from pmdd_b200.writer import FrontierWriter, write_frontier_csv_gz

CASES = [c for c in golden_cases() if "1" in c["methods"]][:10]


def golden_csv_bytes(rec, m=1):
    path = os.path.join(os.path.dirname(rec["dat"]), f"{rec['name']}.m{m}.csv")
    with open(path, "rb") as f:
        return f.read()


@pytest.mark.parametrize("rec", CASES, ids=[c["name"] for c in CASES])
def test_sorted_csv_equals_the_reference_text(rec, tmp_path):
    text = golden_csv_bytes(rec)
    pts = np.array([list(map(int, line.split(","))) for line in text.decode().splitlines()], dtype=np.int32)
    rng = np.random.default_rng(len(pts))
    shuffled = pts[rng.permutation(len(pts))]
    out = str(tmp_path / "f.csv.gz")
    write_frontier_csv_gz(shuffled, out)
    with gzip.open(out, "rb") as f:
        assert f.read() == text


@pytest.mark.skipif(not oracle.have_ref(3), reason="reference binary not built")
def test_bytes_equal_the_reference_binarys_own_file(tmp_path):
    rec = next(c for c in golden_cases() if c["name"] == "kp3_n40_s0")
    ref_out = str(tmp_path / "ref.csv.gz")
    subprocess.run([oracle.ref_binary(3), rec["dat"], "1", "1", "0", "--backend", "cpu", "--frontier-out", ref_out],
                   check=True, capture_output=True)
    dd = DecisionDiagram.from_file(rec["dat"], 1, 3)
    pts = oracle.enumerate(dd, 1)
    ours = str(tmp_path / "ours.csv.gz")
    write_frontier_csv_gz(pts[::-1].copy(), ours)
    with gzip.open(ref_out, "rb") as a, gzip.open(ours, "rb") as b:
        assert a.read() == b.read()


def test_int64_points_and_empty_frontier(tmp_path):
    pts = np.array([[2**40, -5], [-(2**35), 7], [3, 3]], dtype=np.int64)
    out = str(tmp_path / "w.csv.gz")
    write_frontier_csv_gz(pts, out)
    with gzip.open(out, "rt") as f:
        assert f.read() == f"{-(2**35)},7\n3,3\n{2**40},-5\n"
    empty = str(tmp_path / "e.csv.gz")
    write_frontier_csv_gz(np.zeros((0, 3), dtype=np.int32), empty)
    with gzip.open(empty, "rb") as f:
        assert f.read() == b""


def test_unsorted_write_keeps_the_given_order(tmp_path):
    pts = np.array([[3, 1], [1, 3], [2, 2]], dtype=np.int32)
    out = str(tmp_path / "u.csv.gz")
    write_frontier_csv_gz(pts, out, sort=False)
    with gzip.open(out, "rt") as f:
        assert f.read() == "3,1\n1,3\n2,2\n"
    assert pts.tolist() == [[3, 1], [1, 3], [2, 2]]  # the caller's array is untouched


def test_async_writer_many_results(tmp_path):
    rng = np.random.default_rng(3)
    jsonl = str(tmp_path / "stats.jsonl")
    want = {}
    with FrontierWriter(threads=4) as w:
        for i in range(240):
            d = int(rng.integers(1, 8))
            n = int(rng.integers(0, 400))
            dtype = np.int64 if i % 7 == 0 else np.int32
            pts = rng.integers(-1000, 10**6, size=(n, d)).astype(dtype)
            path = str(tmp_path / f"r{i}.csv.gz")
            rec = json.dumps({"request": i, "num_solutions": n, "pad": "x" * int(rng.integers(0, 3000))})
            w.submit(pts, path, jsonl, rec)
            pts[:] = 0  # the writer copied the points at submit
            want[i] = (path, n)
        assert w.flush() == 240
        assert w.pending() == 0
    for i, (path, n) in want.items():
        with gzip.open(path, "rt") as f:
            lines = f.read().splitlines()
        assert len(lines) == n
        rows = [tuple(map(int, line.split(","))) for line in lines]
        assert rows == sorted(rows)
    with open(jsonl) as f:
        recs = [json.loads(line) for line in f]
    assert sorted(r["request"] for r in recs) == list(range(240))


def test_async_writer_reports_failures(tmp_path):
    with FrontierWriter(threads=2) as w:
        w.submit(np.ones((3, 2), dtype=np.int32), str(tmp_path / "missing_dir" / "x.csv.gz"))
        w.submit(np.ones((3, 2), dtype=np.int32), str(tmp_path / "ok.csv.gz"))
        with pytest.raises(OSError, match="1 result"):
            w.flush()
        assert w.flush() == 0  # counters reset after a flush
        with pytest.raises(ValueError):
            w.submit(np.ones((1, 2), dtype=np.int32))  # no output path
        with pytest.raises(ValueError):
            w.submit(None, None, str(tmp_path / "s.jsonl"), "two\nlines")
    assert os.path.exists(tmp_path / "ok.csv.gz")


def test_destroy_writes_what_is_queued(tmp_path):
    w = FrontierWriter(threads=1)
    for i in range(50):
        w.submit(np.full((100, 3), i, dtype=np.int32), str(tmp_path / f"q{i}.csv.gz"))
    w.close()
    for i in range(50):
        with gzip.open(tmp_path / f"q{i}.csv.gz", "rt") as f:
            assert len(f.read().splitlines()) == 100
