"""CPU: the reference arm of bench.py describes the same workload as the
device arm.

`bench.py --impl reference` times the reference's own CPU MD (the reference
library compiled from its sources into oracle/_ref) on the 20,566-atom
workload.  Its JSON line must carry the device arm's `config` unchanged (the
two lines are compared as one workload), the same warm-up plan, and its
thread count in `cpu_baseline.cores` rather than in `config`.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_driver_timing")),
                    reason="the reference is not compiled here (oracle/Makefile ref)")
def test_reference_arm_line_matches_the_device_arm():
    import bench
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["config"] == bench.headline_config(line["config"]["atoms"], 1)
    assert line["warmup"] == sum(bench.warmup_plan(3, 2))
    assert line["cpu_baseline"]["cores"] == 1 and line["cpu_baseline"]["kind"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "ns/day" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
