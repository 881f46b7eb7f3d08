"""bench.py's reference arm on the CPU: the line it prints keeps the bench contract (metric, unit,
config identical to the GPU arm's, cpu_baseline, e2e without host-device bytes), and the process
that times the reference never maps this package's CUDA library, so the reference's numbers come
from the reference alone (its operator and its FillRandom, compiled from its own headers)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import io, json, sys, contextlib
sys.path.insert(0, ROOT)
import bench
args = bench.parse_args(["--impl", "reference", "--steps", "2", "--warmup", "1"])
out = io.StringIO()
with contextlib.redirect_stdout(out):
    rc = bench.run_reference(args)
maps = open("/proc/self/maps").read()
print(json.dumps({"rc": rc, "line": out.getvalue().strip().splitlines()[-1],
                  "libdgop_mapped": "libdgop" in maps, "config": bench.workload_config(1)}))
"""


def test_reference_arm_line_and_isolation():
    sys.path.insert(0, ROOT)
    from oracle.bindings import have_reference
    if not have_reference():
        pytest.skip("oracle/_ref is not built (no reference checkout here)")
    r = subprocess.run([sys.executable, "-c", SCRIPT.replace("ROOT", repr(ROOT))], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["rc"] == 0
    assert not res["libdgop_mapped"]
    line = json.loads(res["line"])
    assert line["impl"] == "reference"
    assert line["unit"] == "GDoF/s" and line["higher_is_better"] is True and line["value"] > 0
    assert line["config"] == res["config"]
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "GDoF/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
