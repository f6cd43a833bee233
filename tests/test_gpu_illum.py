"""Source illumination (reference illum, src/util/fd.cpp:275-339, and
illumPlane, :720-786) on the GPU: bit for bit against the oracle restatement
(pinned to the compiled reference by tests/test_oracle.py), single shots and a
ragged batch."""
import numpy as np
import pytest

import oracle as O
from helpers import golden_cases, golden_ids
from seis_b200 import Shot, fd
from seis_b200._lib import OP_ILLUM, batch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("g", golden_cases(), ids=golden_ids())
def test_illum_golden_bit_exact(ctx, g):
    s = g.shot
    got = fd.illum(s.dt, s.dx, s.dz, s.nt, s.ndel, s.nx, s.nz, s.pml, s.sx, s.sz, g.wav, g.vel,
                   ctx=ctx)
    want = O.illum(s, g.wav, g.vel)
    assert np.array_equal(got, want)
    assert np.abs(want).max() > 0


def test_illum_ragged_batch(ctx):
    rng = np.random.default_rng(5)
    shots, wavs, vels = [], [], []
    for nx, nz, pml in ((70, 40, 12), (45, 61, 3), (130, 33, 20)):
        s = Shot(nx=nx, nz=nz, pml=pml, nt=150, ndel=30, sx=nx // 2, sz=2, dt=1e-3, dx=10.0,
                 dz=10.0, gz=np.zeros(nx, np.int32))
        shots.append(s)
        wavs.append(O.ricker(s.dt, 20.0, s.ndel, s.NT))
        vels.append((1600 + 1500 * rng.random((nx, nz))).astype(np.float32))
    outs = batch(ctx, OP_ILLUM, shots, wavs, vels)
    for s, w, v, o in zip(shots, wavs, vels, outs):
        assert np.array_equal(o, O.illum(s, w, v))


@pytest.mark.parametrize("g", golden_cases(), ids=golden_ids())
def test_illum_plane_golden_bit_exact(ctx, g):
    s = g.shot
    rng = np.random.default_rng(9)
    sou = np.outer(rng.standard_normal(s.nx), g.wav).astype(np.float32)
    got = fd.illum_plane(s.dt, s.dx, s.dz, s.nt, s.ndel, s.nx, s.nz, s.pml, s.sz, g.vel, sou,
                         ctx=ctx)
    want = O.illum_plane(s, sou, g.vel)
    assert np.array_equal(got, want)
    assert want.max() > 0
