"""Host-side helpers of bench.py that its JSON line depends on, checked on the CPU: the
knapsack text parser that feeds device DD construction, the upload byte count behind
e2e.h2d_bytes_per_step, the roofline peak lookup, and the clocks summary that decides
whether a run saw a throttle reason."""
import json

import numpy as np

import bench
import pmdd_b200 as P
from pmdd_b200 import instances


def test_knapsack_text_parses_back_to_the_generator_arrays():
    for n, d, seed in ((20, 3, 0), (60, 3, 5), (25, 7, 1), (1, 1, 2)):
        prof, w, cap = bench.kp_arrays_from_text(instances.knapsack_text(n, d, seed))
        want_p, want_w, want_c = instances.knapsack_arrays(n, d, seed)
        assert np.array_equal(prof, np.asarray(want_p)) and np.array_equal(w, np.asarray(want_w))
        assert cap == int(want_c)


def test_upload_bytes_are_the_dd_arrays():
    for ptype, text in ((1, instances.knapsack_text(30, 3, 4)), (2, instances.setpacking_text(40, 12, 3, 1)),
                        (3, instances.tsp_text(8, 4, 2))):
        dd = P.DecisionDiagram.from_text(text, ptype, 4 if ptype == 3 else 3)
        arrays = [a for a in dd.arrays().values() if a is not None]
        assert bench.dd_bytes(dd) == sum(a.nbytes for a in arrays)


def test_peak_comes_from_the_measured_file(tmp_path, monkeypatch):
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6557.4, "bf16_tflops": 1500.0}))
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.read_peaks() == (6557.4, "measured")
    (tmp_path / "MEASURED_PEAKS.json").unlink()
    assert bench.read_peaks() == (6650.0, "fallback")


def test_clock_summary_reports_median_and_throttle_reasons(tmp_path):
    rows = [
        "0, 1965, 1965, 640.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 801.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1700, 1965, 990.5, 0x0000000000000008, Active, Not Active, Not Active, Not Active",
        "garbage line",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    s = bench.ClockSampler(0)
    s.path = str(tmp_path / "clocks.csv")
    (tmp_path / "clocks.csv").write_text("\n".join(rows) + "\n")
    out = s.summary()
    assert out == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["hw_slowdown", "sw_power_cap"], "samples": 3}
    assert not (tmp_path / "clocks.csv").exists()  # the sample file is removed


def test_clock_summary_without_samples(tmp_path):
    s = bench.ClockSampler(0)
    s.path = str(tmp_path / "missing.csv")
    assert s.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
