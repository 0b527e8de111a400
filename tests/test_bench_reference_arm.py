"""bench.py's reference arm on the CPU: it runs, prints one JSON line with the contract's
keys and the same workload config as the GPU arm, and never loads the product library
(its corpus comes from oracle/sample_corpus.py, its sweeps from the oracle)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
try:
    runpy.run_path("bench.py", run_name="__main__")
finally:
    maps = open("/proc/self/maps").read()
    print(json.dumps({"product_loaded": "liblda_b200" in maps, "oracle_loaded": "liblda_oracle" in maps}))
"""


def test_reference_arm_line_and_isolation():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    line, probe = lines[0], lines[-1]
    assert probe == {"product_loaded": False, "oracle_loaded": True}
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    # the same config dict the GPU arm prints for the default preset
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == bench.workload_config("c1")
    # a step is a whole sweep of the sample, so the time it reports is time spent sweeping
    assert line["ms_per_step"] * line["steps"] < 120_000
