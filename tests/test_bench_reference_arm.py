"""The reference arm of bench.py on the CPU: the reference's own CPU backend
(oracle/_ref) timed on the GPU arm's timed steps from the state after the
warm-up steps (stepped here by the reference itself, as no GPU is present),
printed as one JSON line with the metric, unit and config of the GPU arm."""

import json
import subprocess
import sys
from pathlib import Path

import pytest

from oracle.native import REFERENCE_PATH

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(not REFERENCE_PATH.exists(), reason="the reference library is not built")
def test_reference_arm_line():
    out = subprocess.run(
        [sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "3", "--cells", "2000"],
        cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["steps"] == 2 and line["warmup"] == 3 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert "timed steps 3..4" in line["cpu_baseline"]["sample"]
    assert "after 3 warm-up steps" in line["cpu_baseline"]["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
