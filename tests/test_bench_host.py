"""Host logic of the benchmark (no GPU): the algorithmic byte model behind the
roofline, the peak it divides by, and the workload parameters."""
import json
import math
import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402


def test_algorithmic_bytes_neumann_and_periodic():
    a = bench.algorithmic_bytes("neumann", 256, 1, "fp32")
    r = 4 * 256 ** 3                       # one real field R
    assert a == {"pencil": 4 * r, "plane": 2 * r, "field": r}
    assert a["plane"] == 134217728         # the bench line's algorithmic_bytes_per_launch
    p = bench.algorithmic_bytes("periodic", 128, 1, "fp64")
    h = 2 * 8 * 128 * 128 * 65             # one half spectrum H
    assert p["pencil"] + p["plane"] == 6 * h
    b = bench.algorithmic_bytes("periodic", 64, 64, "fp32")
    assert b["field"] == 64 * 2 * 4 * 64 * 64 * 33


def test_peak_from_measured_file_or_fallback(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6450.0}))
    assert bench.peaks() == (6450.0, "measured")


def test_workload_parameters():
    p = bench.params_for("neumann256")
    assert (p.n, p.batch, p.boundary, p.precision) == (256, 1, "neumann", "fp32")
    assert p.dt == 0.05 and p.eps == -0.75 and p.beta == 2.0 and p.gamma == 1.0 and p.q0 == 1.0
    assert p.dx == pytest.approx(2 * math.pi / 8)
    assert bench.params_for("neumann256", "fp64").precision == "fp64"
    q = bench.params_for("batch64")
    assert q.batch == 64 and len(q.eps_per_replica) == 64
    assert q.eps_per_replica[0] == pytest.approx(-0.9) and q.eps_per_replica[-1] == pytest.approx(-0.5)
    assert "neumann 256^3 x1" in bench.workload_label("neumann256")


def test_workload_ics_are_seeded():
    import numpy as np
    a = bench.make_ic("noise", 16, 3, 0.785, seed=2)
    assert a.shape == (3, 16, 16, 16) and np.array_equal(a, bench.make_ic("noise", 16, 3, 0.785, seed=2))
    h = bench.make_ic("hyperboloid", 16, 1, 0.785)
    assert h.shape == (16, 16, 16)


class _FakeNvml:
    """Read-only NVML stand-in: SM clock and clocks-event reasons per call."""
    NVML_CLOCK_SM = 1

    def __init__(self, clocks, reasons):
        self.clocks, self.reasons, self.i = clocks, reasons, 0

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        return self.clocks[self.i % len(self.clocks)]

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        v = self.reasons[self.i % len(self.reasons)]
        self.i += 1
        return v


def test_clock_sampler_median_and_reasons(monkeypatch):
    import time
    fake = _FakeNvml([1965, 1950, 1965], [0x0, 0x4, 0x0])
    s = bench.ClockSampler(0, period=0.002)
    monkeypatch.setattr(s, "_handle", lambda: (fake, object()))
    s.start()
    s.begin()
    time.sleep(0.05)
    s.end()
    rec = s.stop()
    assert rec["sm_max_mhz"] == 1965 and rec["sm_mhz"] in (1950, 1965, 1957.5)
    assert rec["reasons"] == ["sw_power_cap"] and rec["samples"] >= 3


def test_clock_sampler_without_nvml_reports_nothing(monkeypatch):
    s = bench.ClockSampler(0)

    def broken():
        raise RuntimeError("no NVML")
    monkeypatch.setattr(s, "_handle", broken)
    s.start()
    assert s.stop() is None


def _run_bench(args, env_extra):
    import os
    import subprocess
    env = dict(os.environ, **env_extra)
    root = Path(__file__).resolve().parents[1]
    return subprocess.run([sys.executable, str(root / "bench.py"), *args], capture_output=True, text=True,
                          env=env, timeout=300)


def test_reference_arm_rank0_prints_one_line_other_ranks_nothing():
    args = ["--impl", "reference", "--workload", "periodic128", "--steps", "1", "--warmup", "3"]
    r1 = _run_bench(args, {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r1.returncode == 0 and r1.stdout.strip() == ""
    r0 = _run_bench(args, {"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"})
    assert r0.returncode == 0, r0.stderr[-2000:]
    lines = [ln for ln in r0.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["higher_is_better"] is True and d["metric"] == bench.METRIC
    # the arm runs the warm-up and timed steps it was asked for
    assert d["steps"] == 1 and d["warmup"] == 3


def test_warmup_below_three_is_refused():
    r = _run_bench(["--impl", "reference", "--warmup", "2"], {"RANK": "1"})
    assert r.returncode != 0 and "--warmup must be >= 3" in r.stderr
