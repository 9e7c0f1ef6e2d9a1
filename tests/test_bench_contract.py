"""The bench's reference arm runs on the host cores alone: its JSON line
carries the keys of the bench contract, on a small field."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    oracle_ref = os.path.join(ROOT, "oracle", "_ref", "libszp_ref.so")
    oracle_lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not (os.path.exists(oracle_ref) or os.path.exists(oracle_lib)):
        pytest.skip("oracle not built")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--side", "64",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert "workload" in line["config"]
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and "the whole" in cb["sample"]
    assert cb["one_thread"]["value"] > 0 and len(cb["slab_step_seconds"]) == 1 and cb["slab_value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
