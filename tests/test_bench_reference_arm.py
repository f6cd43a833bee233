"""The benchmark's reference arm (the reference's own CPU forward and adjoint,
compiled from its sources) prints one JSON line with the contract's keys, on
the GPU arm's workload.  Host-only."""
import json
import os
import subprocess
import sys

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True,
                         text=True, timeout=600, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup",
              "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "Gcell-updates/s"
    assert d["config"]["workload"] == "lsrtm_iter" and d["config"]["shots_per_gpu"] == 32
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "reference"
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
