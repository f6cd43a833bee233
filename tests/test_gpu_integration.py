"""The fd.h drop-in of INTEGRATION.md, built by oracle/shim/build_integration.py
into oracle/_ref/fd_shim_check (the reference's fd.h signatures and MyAlloc
arrays, linked with libseisfd.so), run on the golden cases: its gathers and
images must be the reference's, bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from helpers import golden_cases, golden_ids

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "fd_shim_check")
CASES = golden_cases()


@pytest.mark.skipif(not os.path.exists(EXE), reason="drop-in not built (needs the reference)")
@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_drop_in_matches_reference(tmp_path, g):
    s = g.shot
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([s.nx, s.nz, s.pml, s.nt, s.ndel, s.sx, s.sz], np.int32).tofile(f)
        np.array([s.dt, s.dx, s.dz], np.float32).tofile(f)
        np.asarray(s.gz, np.int32).tofile(f)
        for a in (g.wav, g.vel, g.dv, g.rec):
            np.ascontiguousarray(a, np.float32).tofile(f)
    subprocess.run([EXE, str(inp), str(out)], check=True, timeout=300)
    r = np.fromfile(out, np.float32)
    n_rec, n_img = s.nx * s.nt, s.nx * s.nz
    sizes = [n_rec, n_rec, n_img, n_img, n_img]
    assert r.size == sum(sizes)
    parts = np.split(r, np.cumsum(sizes)[:-1])
    rec, born, img, ss, img_true = (p.reshape(s.nx, -1) for p in parts)
    assert np.array_equal(rec, g.rec)
    assert np.array_equal(born, g.born)
    assert np.array_equal(img, g.img)
    assert np.array_equal(ss, O.illum(s, g.wav, g.vel))
    assert np.array_equal(img_true, O.rtm_true(s, g.wav, g.vel, g.rec))
