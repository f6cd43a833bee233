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
    """One JSON line with the contract's keys and the GPU arm's config; the
    process never imports this package nor maps its CUDA library."""
    probe = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', "
             "'--warmup', '0']; runpy.run_path('bench.py', run_name='__main__'); "
             "maps = open('/proc/self/maps').read(); "
             "assert 'libseisfd' not in maps, 'product library mapped'; "
             "assert not [m for m in sys.modules if m.split('.')[0] == 'seis_b200'], 'package imported'")
    out = subprocess.run([sys.executable, "-c", probe], cwd=ROOT, capture_output=True,
                         text=True, timeout=600, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup",
              "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "Gcell-updates/s"
    assert d["config"]["workload"] == "lsrtm_large" and d["config"]["shots_per_gpu"] == 8
    assert d["config"]["shot_indices_rank0"] == [0, 32, 64, 96, 128, 160, 192, 224]
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "reference"
    assert d["cpu_baseline"]["cores"] >= 1 and d["cpu_baseline"]["cpu"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_both_arms_share_the_config():
    """The config the GPU arm starts from is the reference arm's (the GPU arm
    adds measured fields of its own)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    full, mine, _ = b.workload("lsrtm_large", 0, 1)
    sv = full.subset(mine)
    c = b.config_of("lsrtm_large", full, sv, 1)
    assert c["apertures_rank0"] == [2055, 2508, 1137, 3347, 2740, 2093, 1356, 2384]
    assert c["nt"] == 8000 and c["ndel"] == 120 and c["grid"].startswith("4000x1000")
