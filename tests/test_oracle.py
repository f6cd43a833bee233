"""The C restatement in oracle/ against the reference's own outputs.

The golden fixtures were produced by the reference's fd.cpp compiled
unmodified (tests/golden/make_golden.py).  The single-precision restatement
must reproduce them exactly; the double-precision build must agree to FP32
rounding level."""
import numpy as np
import pytest

import oracle as O
from helpers import golden_cases, golden_ids, rel_l2
from seis_b200 import Shot

CASES = golden_cases()


@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_helpers_exact(g):
    s = g.shot
    assert np.array_equal(O.ricker(s.dt, g.fr, s.ndel, s.NT), g.wav)
    assert np.array_equal(O.set_abs(s.nz, s.nx, s.pml), g.abs)
    assert np.array_equal(O.set_vel(g.vel, s.pml), g.velpml)
    assert np.array_equal(O.hilbert(g.hil_in), g.hil_out)


@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_modeling_exact(g):
    assert np.array_equal(O.modeling(g.shot, g.wav, g.vel), g.rec)


@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_born_exact(g):
    assert np.array_equal(O.born(g.shot, g.wav, g.vel, g.dv), g.born)


@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_rtm_exact(g):
    assert np.array_equal(O.rtm(g.shot, g.wav, g.vel, g.rec), g.img)


@pytest.mark.parametrize("g", CASES[:2], ids=golden_ids()[:2])
def test_f64_build_tracks_f32(g):
    """The FP64 oracle is the same code in double: FP32 gathers sit within
    FP32 rounding of it."""
    r64 = O.modeling(g.shot, g.wav.astype(np.float64), g.vel, prec="f64")
    assert rel_l2(g.rec, r64) < 1e-5
    b64 = O.born(g.shot, g.wav.astype(np.float64), g.vel, g.dv, prec="f64")
    assert rel_l2(g.born, b64) < 1e-4


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
def test_restatement_matches_reference_random():
    """Fresh random case, both implementations run here."""
    from seis_b200 import Shot
    rng = np.random.default_rng(99)
    nx, nz = 33, 29
    s = Shot(nx=nx, nz=nz, pml=7, nt=90, ndel=11, sx=16, sz=3, dt=8e-4, dx=7.5, dz=9.0,
             gz=rng.integers(0, nz, nx))
    vel = (1600 + 2000 * rng.random((nx, nz))).astype(np.float32)
    dv = rng.standard_normal((nx, nz)).astype(np.float32)
    wav = O.ricker(s.dt, 30.0, s.ndel, s.NT, impl="ref")
    rec = O.modeling(s, wav, vel, impl="ref")
    assert np.array_equal(O.modeling(s, wav, vel), rec)
    assert np.array_equal(O.born(s, wav, vel, dv), O.born(s, wav, vel, dv, impl="ref"))
    assert np.array_equal(O.rtm(s, wav, vel, rec), O.rtm(s, wav, vel, rec, impl="ref"))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_illum_restatement_matches_reference(g):
    """illum (src/util/fd.cpp:275-339): the C restatement bit for bit."""
    assert np.array_equal(O.illum(g.shot, g.wav, g.vel), O.illum(g.shot, g.wav, g.vel, impl="ref"))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_born_plane_restatement_matches_reference(g):
    """forwordPlane (src/util/fd.cpp:178-274): the C restatement bit for bit."""
    rng = np.random.default_rng(1)
    sou = np.outer(rng.standard_normal(g.shot.nx), g.wav).astype(np.float32)
    gz = int(g.shot.gz[0])
    assert np.array_equal(O.born_plane(g.shot, sou, g.vel, g.dv, gz),
                          O.born_plane(g.shot, sou, g.vel, g.dv, gz, impl="ref"))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_illum_plane_restatement_matches_reference(g):
    """illumPlane (src/util/fd.cpp:720-786): the C restatement bit for bit."""
    rng = np.random.default_rng(4)
    sou = np.outer(rng.standard_normal(g.shot.nx), g.wav).astype(np.float32)
    want = O.illum_plane(g.shot, sou, g.vel, impl="ref")
    assert np.array_equal(O.illum_plane(g.shot, sou, g.vel), want)
    assert want.max() > 0


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_rtm_plane_restatement_matches_reference(g):
    """adjointPlane (src/util/fd.cpp:787-921): the C restatement bit for bit,
    with the gather's last ndel + 2 samples zero (the reference reads them at
    negative indices, fd.cpp:834, :873; the restatement skips those)."""
    s = g.shot
    rng = np.random.default_rng(3)
    sou = np.outer(rng.standard_normal(s.nx), g.wav).astype(np.float32)
    rec = rng.standard_normal((s.nx, s.nt)).astype(np.float32)
    rec[:, s.nt - (s.ndel + 2):] = 0.0
    gz = int(s.gz[0])
    assert np.array_equal(O.rtm_plane(s, sou, g.vel, rec, gz),
                          O.rtm_plane(s, sou, g.vel, rec, gz, impl="ref"))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_rtm_true_restatement_matches_reference(g):
    """rtm_true (src/util/fd.cpp:924-1052): the C restatement bit for bit."""
    assert np.array_equal(O.rtm_true(g.shot, g.wav, g.vel, g.rec),
                          O.rtm_true(g.shot, g.wav, g.vel, g.rec, impl="ref"))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("g", CASES[:2], ids=golden_ids()[:2])
def test_rtm_updown_restatement_matches_reference(g):
    """adjointUpDown (src/util/fd.cpp:340-590): image and all four components
    of the C restatement bit for bit."""
    wavh = O.hilbert(g.wav, 30)
    img, comp = O.rtm_updown(g.shot, g.wav, wavh, g.vel, g.rec)
    rimg, rcomp = O.rtm_updown(g.shot, g.wav, wavh, g.vel, g.rec, impl="ref")
    assert np.array_equal(img, rimg)
    assert np.array_equal(comp, rcomp)
    assert np.abs(comp).max(axis=(1, 2)).min() > 0


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
def test_reference_scheme_unstable_above_courant_053():
    """The reference's own modeling (fd.cpp:15-80) grows without bound at a
    Courant number v dt / dx of 0.55 -- below the 0.5546 limit of its interior
    8th-order update, so the growth comes from its boundary treatment -- and
    decays at 0.45; the restatement follows it bit for bit in both regimes."""
    amp = {}
    for v in (5500.0, 4500.0):
        s = Shot(nx=60, nz=50, pml=20, nt=3000, ndel=60, sx=30, sz=1, dt=5e-4, dx=5.0, dz=5.0,
                 gz=np.full(60, 1, np.int32))
        vel = np.full((s.nx, s.nz), v, np.float32)
        wav = O.ricker(s.dt, 25.0, s.ndel, s.NT)
        ref = O.modeling(s, wav, vel, impl="ref")
        assert np.array_equal(O.modeling(s, wav, vel), ref)
        amp[v] = np.abs(ref[:, -500:]).max() / np.abs(ref[:, :1000]).max()
    assert amp[5500.0] > 1e3
    assert amp[4500.0] < 1e-3
