"""CPU tests of bench.py's reference arm: it runs on the host only, prints one JSON line
with the contract's keys and the impl marker."""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline",
        "dtype", "data", "config", "cpu_baseline", "e2e"}


@pytest.mark.parametrize("workload", ["return_map", "rve_path", "rno_train", "implicit_fe2", "rno_energy"])
def test_reference_arm_prints_one_contract_line(workload: str) -> None:
    cmd = [sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--workload", workload, "--steps", "1",
           "--warmup", "1"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [line for line in out.stdout.splitlines() if line.strip().startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert KEYS <= set(rec) and rec["impl"] == "reference" and rec["value"] > 0
    assert rec["cpu_baseline"]["kind"] == "port" and rec["cpu_baseline"]["cores"] >= 1
    assert rec["e2e"]["value"] == rec["value"]
