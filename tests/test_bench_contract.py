"""bench.py's reference arm (the CPU restatement on a bounded sample) prints
one JSON line with the keys the benchmark contract asks for; it needs no
GPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                          "--no-cpu-trend"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    r = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in r, k
    assert r["impl"] == "reference" and r["value"] > 0 and r["higher_is_better"] is True
    assert r["cpu_baseline"]["kind"] == "port" and r["cpu_baseline"]["cores"] >= 1
    assert r["e2e"]["h2d_bytes_per_step"] == 0 and r["e2e"]["value"] == r["value"]


def test_cpu_trend_extrapolation():
    """Each stage fitted as t = a n^k through the two measured points: a stage
    that is linear in n extrapolates linearly, a quadratic one quadratically."""
    sys.path.insert(0, ROOT)
    import bench
    calls = {}

    def fake_run(name, steps, warmup, nth):
        calls[name] = steps
        return 8 * 100, 72.0, {"lin": 8.0, "quad": 64.0}

    orig = bench.cpu_oracle_run
    bench.cpu_oracle_run = fake_run
    try:
        t = bench.cpu_trend((100, 2.0, {"lin": 1.0, "quad": 1.0}), 4, 64 * 100)
    finally:
        bench.cpu_oracle_run = orig
    assert calls == {bench.CPU_TREND: 1}
    e = t["extrapolated"]
    assert abs(e["stage_exponents"]["lin"] - 1.0) < 1e-9 and abs(e["stage_exponents"]["quad"] - 2.0) < 1e-9
    assert abs(e["stage_s"]["lin"] - 64.0) < 0.1 and abs(e["stage_s"]["quad"] - 4096.0) < 0.1
    assert "not measured" in e["note"]
