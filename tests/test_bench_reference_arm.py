"""`bench.py --impl reference` on the CPU: the reference's own IntersectBvh
(compiled by oracle/Makefile) times the traversal workload and prints the
bench line's keys; under a multi-rank launch only rank 0 prints."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402


def _run(extra_env: dict) -> subprocess.CompletedProcess:
    env = dict(os.environ, **extra_env)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0", "--rays", "65536"], capture_output=True, text=True, env=env,
                          timeout=600, cwd=ROOT)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref is not built")
def test_reference_arm_line():
    res = _run({"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"})
    assert res.returncode == 0, res.stderr[-2000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "Mrays/s traversal" and line["unit"] == "Mrays/s"
    assert line["higher_is_better"] is True
    assert line["config"]["rays_per_step"] == 65536
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["cpu_baseline"]["value"] == line["value"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    res = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert res.returncode == 0, res.stderr[-2000:]
    assert res.stdout.strip() == ""
