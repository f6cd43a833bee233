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


def test_driver_plane_pipeline(ctx, tmp_path):
    """planeWavePrepare, then adjointPlane_MPI and illumPlane_MPI through the shot driver, against
    the restatement on the files the preparation wrote."""
    from seis_b200 import Shot
    from seis_b200.driver import Driver
    from test_plane_prepare import DELAYCAL, NT, NX, NZ, write_survey
    param = write_survey(tmp_path, tmp_path / "W", np.random.default_rng(4))
    v0 = np.broadcast_to(1800.0 + 20.0 * np.arange(NZ), (NX, NZ)).astype(np.float32)
    v0.tofile(tmp_path / "v0.bin")
    with Driver(ctx, str(param)) as d:
        d.plane_prepare()
        img = d.rtm_plane()
        ss = d.illum_plane()
        npw = d.params.np
    shot = Shot(nx=NX, nz=NZ, pml=10, nt=NT, ndel=DELAYCAL, sx=NX // 2, sz=1, dt=1e-3, dx=10.0,
                dz=10.0, gz=np.full(NX, 1, np.int32))
    want = np.zeros((NX, NZ), np.float32)
    for k in range(npw):
        sou = np.fromfile(tmp_path / "W" / f"PLANE_S_NEW{k}.dat", np.float32).reshape(NX, NT + DELAYCAL)
        rec = np.fromfile(tmp_path / "W" / f"PLANE_R_NEW{k}.dat", np.float32).reshape(NX, NT)
        im = O.rtm_plane(shot, sou, v0, rec, 1)
        got_k = np.fromfile(tmp_path / "W" / f"IMAGE{k}.dat", np.float32).reshape(NX, NZ)
        assert np.array_equal(got_k, im), k
        want = im + want
    assert np.array_equal(img, want)
    assert np.abs(img).max() > 0
    # illumPlane_MPI: one ILLUM_PLANE<k>.dat per wavenumber
    ss_want = np.zeros((NX, NZ), np.float32)
    for k in range(npw):
        sou = np.fromfile(tmp_path / "W" / f"PLANE_S_NEW{k}.dat", np.float32).reshape(NX, NT + DELAYCAL)
        ill = O.illum_plane(shot, sou, v0)
        got_k = np.fromfile(tmp_path / "W" / f"ILLUM_PLANE{k}.dat", np.float32).reshape(NX, NZ)
        assert np.array_equal(got_k, ill), k
        ss_want = ill + ss_want
    assert np.array_equal(ss, ss_want)
    assert ss.max() > 0
