"""The bench's reference arm (`bench.py --impl reference`: the reference's own CPU solver on
the host cores, the oracle port where that library is absent): one JSON line with the
contract's fields from rank 0, nothing from the other ranks of a multi-rank launch."""
import json
import os
import subprocess
import sys

import pytest

import checkers

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.skipif(not checkers.ref_available(), reason="reference library not built")


def run_arm(**env):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0"], capture_output=True, text=True, timeout=900, cwd=ROOT,
                          env=dict(os.environ, **env))


def test_reference_arm_line():
    out = run_arm()
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "body-steps/s at 65k boxes"
    assert line["unit"] == "body-steps/s" and line["higher_is_better"] is True and line["value"] > 0
    assert line["config"]["bodies_per_gpu"] == 65536 and line["steps"] >= 1
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] >= 1 and cpu["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_are_silent():
    out = run_arm(RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip() == ""
