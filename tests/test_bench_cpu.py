"""bench.py on CPU: the reference arm's (--impl reference) one JSON line
carries the keys the benchmark contract asks for, and under a multi-rank
launch only rank 0 works and prints; the algorithmic bytes and roofline
arithmetic of the HBM-rated stages; the clock-sample summary."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "3", "--n", "100000",
        "--ref-sample", "2000"]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + ARGS, cwd=ROOT,
                          env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_line():
    r = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == d["unit"] == "particle-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 3
    assert d["config"]["workload"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port")
    assert cb["cores"] >= 1 and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def test_stage_bytes_follow_the_scope_formulas():
    bench = _bench()
    n, c = 1_000_000, 292_824
    mixed, fp64 = bench.stage_bytes(n, c, 4), bench.stage_bytes(n, c, 8)
    assert mixed["broad_phase"] == fp64["broad_phase"] == 52 * n + 8 * c
    # N (6 S_p + 30 S), plus the mixed mode's FP32 orientation remainder read
    # and written
    assert mixed["integration"] == 200 * n
    assert fp64["integration"] == 288 * n


def test_stage_report_rates_each_stage_against_the_peak():
    bench = _bench()
    from grains3dgpu_b200 import abi
    per_step = np.zeros(len(abi.PHASES))
    for name, ms in {"hash": 0.015, "sort": 0.017, "cell_start": 0.030, "particle": 0.075,
                     "pair_count": 0.46}.items():
        per_step[abi.PHASES.index(name)] = ms
    n, c, hbm = 1_000_000, 292_824, 6538.6
    out = bench.stage_report(per_step, n, c, 4, hbm)
    b = bench.stage_bytes(n, c, 4)
    for stage, ms in (("broad_phase", 0.062), ("integration", 0.075), ("pair_count", 0.46)):
        assert abs(out[stage]["ms"] - ms) < 1e-9
        gbs = b[stage] / (ms * 1e-3) / 1e9
        assert abs(out[stage]["achieved_gbs"] - gbs) <= 0.05
        assert abs(out[stage]["frac_of_measured_hbm"] - gbs / hbm) <= 5e-5


def test_clocks_summary(tmp_path):
    bench = _bench()
    p = tmp_path / "clocks.csv"
    rows = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1965, 1965, 800.0, 0x0, Not Active, Not Active, Not Active, Not Active",
            "1, 900, 1965, 100.0, 0x0, Active, Not Active, Not Active, Not Active"]
    p.write_text("\n".join(rows) + "\n")
    got = bench.clocks_summary(str(p), 0)
    assert got == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"]}
    assert bench.clocks_summary(str(tmp_path / "missing.csv"), 0)["reasons"] == ["unsampled"]
