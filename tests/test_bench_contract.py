"""bench.py's reference arm on the CPU: one JSON line with the contract's keys,
the requested warm-up honoured, and the end-to-end figure equal to the value
(the CPU path copies nothing between host and device)."""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run(
        [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "water-2652",
         "--steps", "2", "--warmup", "4", "--cpu-budget", "1"],
        cwd=ROOT, capture_output=True, text=True, timeout=300, check=True).stdout
    lines = [line for line in out.splitlines() if line.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["metric"] == "ns/day" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 4 and d["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1 and "warm-up" in d["cpu_baseline"]["sample"]
    assert d["cpu_baseline"]["host_cpu"]["nproc"] >= 1
    bench = load_bench()
    assert d["config"] == bench.workload_config("water-2652", 1, 2)


def load_bench():
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_default_workload_is_the_batched_ensemble_and_both_arms_describe_it_alike():
    """The default line is the metric's configuration: the 64-system ensemble,
    batched against plain engines.  Its `config` comes from one function in
    both arms, from the same arguments, so the two lines name the same
    workload; and the reference arm's sampler takes every system at least once
    in K steps."""
    bench = load_bench()
    assert bench.default_config() == "ensemble-64"
    cfg = bench.workload_config("ensemble-64", 1, 20)
    assert cfg["systems"] == 64 and 2000 * 64 < cfg["atoms"] < 30000 * 64
    assert json.loads(json.dumps(cfg)) == cfg
    seen = set()
    sampler = bench.EnsembleSampler([(None, None)] * 64, threads=1, per=-(-64 // 20))
    for _ in range(20):
        for _ in range(sampler.per):
            seen.add(sampler.cursor % 64)
            sampler.cursor += 1
    assert seen == set(range(64))
