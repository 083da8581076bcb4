"""The benchmark's output contract on the CPU: the reference arm (the oracle
port on the host cores) prints one JSON line with the keys and units the
GPU arm uses, and the flop accounting matches the documented product count."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_arm_json_line():
    proc = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert proc.returncode == 0, proc.stderr[-2000:]
    line = json.loads(proc.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "rgf_energy_solves_per_s" and line["unit"] == "solves/s"
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["n_gpus"] == 1
    assert line["value"] > 0 and line["dtype"] == "complex128"
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert "nb=64 b=256" in line["config"]["workload"]


@pytest.mark.parametrize("nb,its,units", [(64, (22, 22), 3 + 2 + 63 * 19 + 6 + 2 * (7 * 22 + 1)),
                                          (2, (1, 3), 3 + 2 + 19 + 6 + 8 + 22)])
def test_flop_accounting(nb, its, units):
    """8 b^3 per block product or inverse; 19 per block step with every output
    (6 forward, 13 backward), 5 for the end blocks, 6 for contacts and
    transmission, 7 per Sancho-Rubio iteration + 1 per lead."""
    import bench

    assert bench._flops_per_energy(nb, 256, list(its)) == 8.0 * 256 ** 3 * units
