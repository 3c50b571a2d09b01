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
    assert d["steps"] >= 1 and d["warmup"] >= 3 and d["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1 and "warm-up" in d["cpu_baseline"]["sample"]
