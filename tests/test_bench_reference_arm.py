"""The bench's reference arm on the CPU: `bench.py --impl reference` times
the reference's own solver (oracle/_ref timing build) and prints one JSON
line with the fields of the bench contract (CPU only; skipped where the
reference build is absent)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import bridge  # noqa: E402

needs_timing = pytest.mark.skipif(not bridge.available("libmpmref_timing.so"),
                                  reason="reference build oracle/_ref/libmpmref_timing.so not present")


@needs_timing
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "blockdrop2d", "--steps", "2", "--warmup", "3"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["unit"] == "particle-steps/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["n_gpus"] == 1
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] >= 1 and cpu["value"] == line["value"] and cpu["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "blockdrop2d" and line["config"]["points"] == 144
