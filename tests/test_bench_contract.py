"""bench.py's reference arm on the CPU: one JSON line with the fields the benchmark contract names.

`bench.py --impl reference` times the reference's own C path (compiled from its sources into
oracle/_ref) on the host cores; it needs no GPU, so its output format is checked here on a
one-step run (one bounded sample of the benchmark field's kind)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

REF_LIB = os.path.join(REPO, "oracle", "_ref", "libmkfref.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference C path not built (oracle/_ref)")
def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0", "--no-secondary"], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Gvoxel/s per field (16 thresholds)" and d["unit"] == "Gvoxel/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"] == "grf1024_f64_k16" and d["config"]["thresholds"] == 16
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "Gvoxel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
