"""Plane-wave operators on the GPU, bit for bit against the oracle
restatement (pinned to the compiled reference by tests/test_oracle.py):
forwordPlane (Born with an areal source, src/util/fd.cpp:178-274) and
adjointPlane (RTM of an areal source, :787-921)."""
import numpy as np
import pytest

import oracle as O
from helpers import golden_cases, golden_ids
from seis_b200 import fd

pytestmark = pytest.mark.gpu


def areal_source(s, wav, seed):
    rng = np.random.default_rng(seed)
    return np.outer(rng.standard_normal(s.nx), wav).astype(np.float32)


@pytest.mark.parametrize("g", golden_cases(), ids=golden_ids())
def test_born_plane_golden_bit_exact(ctx, g):
    s = g.shot
    sou = areal_source(s, g.wav, 7)
    gz = int(s.gz[0])
    got = fd.forward_plane(s.dt, s.dx, s.dz, s.nt, s.ndel, s.nx, s.nz, s.pml, s.sz, gz, g.vel, sou,
                           g.dv, ctx=ctx)
    want = O.born_plane(s, sou, g.vel, g.dv, gz)
    assert np.array_equal(got, want)
    assert np.abs(want).max() > 0


@pytest.mark.parametrize("g", golden_cases(), ids=golden_ids())
def test_rtm_plane_golden_bit_exact(ctx, g):
    s = g.shot
    sou = areal_source(s, g.wav, 11)
    rng = np.random.default_rng(12)
    rec = rng.standard_normal((s.nx, s.nt)).astype(np.float32)
    gz = int(s.gz[0])
    got = fd.adjoint_plane(s.dt, s.dx, s.dz, s.nt, s.ndel, s.nx, s.nz, s.pml, s.sz, gz, g.vel, sou,
                           rec, ctx=ctx)
    want = O.rtm_plane(s, sou, g.vel, rec, gz)
    assert np.array_equal(got, want)
    assert np.abs(want).max() > 0
