"""The benchmark's reference arm on the CPU: one JSON line with the keys the benchmark contract
names, and no output from ranks other than 0 (they exit without work)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=e,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


def test_reference_arm_prints_one_contract_line():
    out = run_bench("--impl", "reference", "--steps", "1", "--warmup", "1", "--scale", "0.25",
                    "--cpu-sample-seconds", "2")
    lines = [l for l in out.strip().splitlines() if l.startswith("{")]
    assert len(lines) == 1, out
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["unit"] == "GFLOP/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_stay_silent():
    out = run_bench("--impl", "reference", "--steps", "1", "--warmup", "1", "--scale", "0.25",
                    "--cpu-sample-seconds", "2", env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert not [l for l in out.strip().splitlines() if l.startswith("{")], out


def test_cpu_sample_flop_accounting_matches_the_oracle():
    # the per-A-block pair flops that size the CPU samples add up to the oracle's flop count,
    # on the whole workload and on a sample of its first stored A blocks
    import numpy as np

    import bench
    import oracle
    from shtensor_b200 import workloads as W
    w = W.c1(seed=3, scale=0.25, occupancy=0.4)
    fl = bench.pair_flops_per_a_block(w)
    r = oracle.contract(w.expr, 1.0, bench.host(w.A), bench.host(w.B), 0.0, bench.host(w.C))
    assert np.isclose(fl.sum(), r.flops, rtol=1e-12)
    samp, k, n = bench.sample_workload(w, 0.3 * r.flops)
    assert 0 < k < n
    rs = oracle.contract(samp.expr, 1.0, bench.host(samp.A), bench.host(samp.B), 0.0, bench.host(samp.C))
    assert np.isclose(fl[:k].sum(), rs.flops, rtol=1e-12) and rs.flops >= 0.3 * r.flops


def test_split_roofline_reports_both_ceilings():
    # the split form's line carries its rate against the dense INT8 peak and against the split
    # operand-pipeline ceiling, with the slice products credited as 28 per FP64 flop at 7 slices
    import bench
    peaks = {"int8": 4000.0, "dmma": 40.0, "split_pipe": 2000.0}
    r = bench.roofline_of("split", 1e12, 10.0, peaks, S=7)  # 1 TFLOP in 10 ms
    assert abs(r["fp64_equivalent"]["achieved"] - 100.0) < 1e-9
    assert abs(r["achieved"] - 2800.0) < 1e-9 and abs(r["frac"] - 0.7) < 1e-12
    op = r["operand_pipeline"]
    assert abs(op["frac"] - 1.4) < 1e-12 and op["peak"] == 2000.0 and op["unit"] == "TOPS"
    assert bench.roofline_of("split", 1e12, 10.0, {"int8": 4000.0}, S=7)["operand_pipeline"]["frac"] is None
