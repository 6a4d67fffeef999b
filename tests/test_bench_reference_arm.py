"""bench.py's reference arm: the CPU restatement on a sample of the chip
workload, one JSON line with the contract's keys, and no CUDA library in the
process (the arm runs the oracle and its host trace generator only)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_RUN = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "0", "--cpu-lanes", "8"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("LOADED", "libhw_b200" in maps, "libhw_oracle" in maps)
"""


def test_reference_arm_line_and_libraries():
    r = subprocess.run([sys.executable, "-c", _RUN], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    m = json.loads(lines[-2])
    assert m["impl"] == "reference"
    assert m["metric"] == "ZMW-frames/s" and m["unit"] == "ZMW-frames/s" and m["higher_is_better"]
    assert m["value"] > 0 and m["e2e"]["value"] == m["value"]
    assert m["e2e"]["h2d_bytes_per_step"] == 0 and m["e2e"]["d2h_bytes_per_step"] == 0
    cb = m["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == m["value"] and cb["cores"] >= 1
    # the 8 sample lanes are spread over the workload's 4 pools
    assert "4 pools" in cb["sample"]
    # per-stage CPU times of the sample
    for stage in ("baseline", "histogram", "labeler", "pulses"):
        assert cb["stages"][stage]["ms_per_step"] > 0, stage
    assert lines[-1] == "LOADED False True"
