"""CPU tests of bench.py's bookkeeping: the algorithmic-byte model of the roofline and the JSON line
of our arm (every key of the contract present, values derived as documented). No GPU work."""
import argparse
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _counters(**kw):
    c = dict(histories=100, crossings=1000, scatterings=50, peel_detections=200, rf_stores=300, stats_overflows=0,
             kernel_launches=17, stats_spilled=0)
    c.update(kw)
    return c


def test_algorithmic_bytes_follow_the_unit_costs():
    c = _counters()
    assert bench.algorithmic_bytes(c, 1) == 64 * 1000 + 128 * 50 + 16 * (200 + 300)
    assert bench.trace_algorithmic_bytes(c, 0) == 4 * 1000 + 16 * 300
    assert bench.trace_algorithmic_bytes(c, 2) == 284 * 1000 + 16 * 300
    assert bench.trace_algorithmic_bytes(c, 3) == 84 * 1000 + 16 * 300


def test_result_line_carries_the_contract_keys():
    args = argparse.Namespace(steps=5, warmup=3, precision="fp32", gpus=1)

    class Clk:
        def summary(self):
            return {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": []}

    c = _counters()
    e2e = {"value": 1.0, "unit": "packets/s", "h2d_bytes_per_step": 8, "d2h_bytes_per_step": 16}
    line = bench.result_line(args, "galaxy", 1, 2.0e7, 5000.0, 4000.0, 100, c, 1, 1, Clk(), e2e, 10 ** 8)
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "roofline", "clocks", "e2e", "gpu_launches"):
        assert key in line, key
    rf = line["roofline"]
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in rf, key
    assert line["ms_per_step"] == 1000.0
    # achieved = trace algorithmic bytes per launch / average launch time
    per_launch = bench.trace_algorithmic_bytes(c, 1) / (100 / 5)
    assert abs(rf["achieved"] - per_launch / (40.0 / 1e3) / 1e9) < 1e-9 * rf["achieved"]
    assert abs(rf["frac"] - rf["achieved"] / rf["peak"]) < 1e-12
    assert line["gpu_launches"] == 17 * 5
    assert line["config"]["workload"] == "galaxy" and line["higher_is_better"] is True


def test_max_over_ranks_is_identity_on_one_rank():
    assert bench.max_over_ranks(3.5, 1, 0) == 3.5
