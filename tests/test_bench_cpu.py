"""bench.py's reference arm on the CPU: the reference's own code on a small
graph, one JSON line with the GPU arm's keys and config, every step the full
workload, and no part of this project's library loaded in that process."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_driver")),
                    reason="the reference's CPU code is not built (oracle/_ref)")
def test_reference_arm_runs_the_full_step_without_the_library():
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--scale', '10', '--steps', '2', "
            "'--warmup', '1']; sys.path.insert(0, %r); import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'hc_imported': 'hc' in sys.modules, 'libhc_mapped': 'libhc.so' in maps, "
            "'liboracle_mapped': 'liboracle.so' in maps}))" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
    line, probe = lines[0], lines[1]
    assert line["impl"] == "reference" and line["unit"] == "GTEPS" and line["value"] > 0
    assert len(line["detail"]["step_ms"]) == 2
    assert abs(sum(line["detail"]["step_ms"]) / 2 - line["ms_per_step"]) < 1e-6
    assert line["config"]["num_edges"] > 0 and line["config"]["parallelism"] == "replicas x1"
    assert line["cpu_baseline"]["kind"] == "reference"
    assert probe == {"hc_imported": False, "libhc_mapped": False, "liboracle_mapped": False}
