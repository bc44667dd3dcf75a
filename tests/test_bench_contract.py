"""The JSON line of `bench.py --impl reference` (the CPU arm the GPU arm is
compared with): one line with the benchmark's metric, unit and workload
label, a positive value, a `cpu_baseline` describing the run and an `e2e`
entry without host-device traffic."""

import json
import os
import subprocess
import sys

import bench
from crest_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--cells", "3000"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    j = json.loads(lines[0])
    assert j["metric"] == bench.METRIC and j["unit"] == bench.UNIT and j["impl"] == "reference"
    assert j["value"] > 0 and j["higher_is_better"] is True and j["steps"] == 1 and j["warmup"] == 0
    w = synth.WORKLOADS["1m"]
    # --cells takes a prefix of the named workload; the label states the cells run
    assert j["config"]["workload"] == bench.workload_label(w, 3000)
    assert 0 < j["config"]["cells_after_qc"] <= 3000
    # the reference arm never maps the product library
    assert j["native_so_loaded"] and all(x.startswith("oracle" + os.sep) for x in j["native_so_loaded"])
    cb = j["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == j["value"]
    assert j["e2e"] == {"value": j["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
