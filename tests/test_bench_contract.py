"""The bench's reference arm on the CPU (the oracle as the reference's CPU
path, on a small sample): one JSON line with the driver's keys, for the MVS
line and the drop-in line. The GPU arm's line is checked on a B200."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def reference_line(*extra):
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--particles", "2000", *extra],
                         cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("workload,metric", [("mvs", "MVS particle-steps/s"),
                                             ("dropin", "MVS drop-in particle-steps/s")])
def test_reference_arm_line(workload, metric):
    d = reference_line("--workload", workload)
    assert d["impl"] == "reference" and d["metric"] == metric
    assert d["unit"] == "particle-steps/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == d["value"] and cpu["sample"]
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"]


def test_compact_launch_steps():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.compact_steps([7] + [31] * 147 + [6]) == "7 + 147x31 + 6"
    assert bench.compact_steps([4, 16]) == "4 + 16"
    assert bench.compact_steps([]) == ""
