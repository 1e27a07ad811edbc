"""The reference CLI linked with this engine's adapter, on CPU.

The binary is the reference's own program with the seam file
pmdd_b200/csrc/adapter/cuda_wrappers_pmdd_b200.cpp in place of its CUDA stubs.  Its CPU
backend must still produce the golden frontier (the link replaced nothing else), and
without a usable GPU its GPU backend must fail the reference's way -- exit status 1 and
"Error - GPU backend requested but ..." with this engine's reason.
"""
import gzip
import os
import subprocess

import pytest

from conftest import GOLDEN, ROOT, golden_cases

EXE = os.path.join(ROOT, "oracle", "_ref", "multiobj_nobjs3_pmdd")


def _gpu_present():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(not os.path.exists(EXE), reason="adapter binary not built (make -C oracle adapter REF=...)")
def test_adapter_binary_cpu_backend_and_gpu_error_path(tmp_path):
    rec = next(r for r in golden_cases() if r["name"] == "kp3_n20_s1")
    fout = tmp_path / "f.csv.gz"
    p = subprocess.run([EXE, rec["dat"], "1", "1", "0", "--backend", "cpu", "--frontier-out", str(fout)],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    with gzip.open(fout, "rt") as f, open(os.path.join(GOLDEN, "kp3_n20_s1.m1.csv")) as g:
        assert f.read() == g.read()
    if _gpu_present():
        pytest.skip("a GPU is present: the GPU path is covered by test_gpu_adapter.py")
    p = subprocess.run([EXE, rec["dat"], "1", "1", "0", "--backend", "gpu"], capture_output=True, text=True,
                       timeout=120)
    assert p.returncode == 1
    assert "Error - GPU backend requested but" in p.stdout + p.stderr
