"""The reference's own command-line program on this engine.

oracle/_ref/multiobj_nobjs<N>_pmdd is the reference's unmodified main.cpp, DD
constructors and CPU objects, linked with pmdd_b200/csrc/adapter/cuda_wrappers_pmdd_b200.cpp
in place of its enum/gpu/cuda_stubs.cpp (built by `make -C oracle adapter`).  With
--backend gpu its four seam calls (src/pmdd/enum/gpu/cuda_wrappers.hpp:11-21) run on
libpmdd_gpu.so; the frontier file and the first stdout line must equal the reference
binary's own (the golden fixtures), for both methods, with state dominance and with a
small --max-cand.
"""
import gzip
import os
import subprocess

import pytest

from conftest import GOLDEN, ROOT, golden_cases

pytestmark = pytest.mark.gpu


def adapter_binary(nobjs):
    return os.path.join(ROOT, "oracle", "_ref", f"multiobj_nobjs{nobjs}_pmdd")


def cases():
    out = []
    for rec in golden_cases():
        for m in sorted(rec["methods"]):
            out.append(pytest.param(rec, int(m), id=f"{rec['name']}-m{m}"))
    return out


@pytest.mark.parametrize("rec,method", cases())
def test_reference_cli_on_this_engine(rec, method, tmp_path):
    exe = adapter_binary(rec["nobjs"])
    if not os.path.exists(exe):
        pytest.skip("adapter binary not built (make -C oracle adapter REF=...)")
    extra = []
    sd = 0
    if rec["problem_type"] == 1 and method == 1:
        sd = 1  # knapsack state dominance: same frontier, fewer labels
    if rec["name"].startswith("kp3_n40"):
        extra = ["--max-cand", "20000"]
    fout = tmp_path / "f.csv.gz"
    p = subprocess.run([exe, rec["dat"], str(rec["problem_type"]), str(method), str(sd), "--backend", "gpu",
                        "--frontier-out", str(fout), *extra], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.splitlines()[0] == rec["methods"][str(method)]["stdout_first_line"]
    with gzip.open(fout, "rt") as f:
        got = f.read()
    with open(os.path.join(GOLDEN, f"{rec['name']}.m{method}.csv")) as f:
        assert got == f.read()
