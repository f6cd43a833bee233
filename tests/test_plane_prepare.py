"""Plane-wave preparation (planeWavePrepare, src/lsrtm/inversion.cpp:808-912)
through the shot driver, bit for bit against the same steps composed from the
reference's own compiled pieces (rickerWavelet, harmonic, swapReord): the
phase-encoded sources PLANE_S_NEW<k>.dat and data PLANE_R_NEW<k>.dat.  (The
member itself cannot run here: its file names come from sprintf("%s") of a
std::string, inversion.cpp:667-690, which g++ 13 garbles.)  Also the Hilbert
filter helper against the oracle.  Host only."""
import numpy as np
import pytest

import oracle as O
from seis_b200._lib import lib
from seis_b200.driver import Driver

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference oracle not built")

NX, NZ, NT, DELAY, DELAYCAL = 60, 30, 180, 4, 40


def write_survey(tmp, wdir, rng):
    lines = []
    shots = []
    for sx in (3, 17, 29, 44):
        gx = np.arange(max(0, sx - 12), min(NX, sx + 15))
        shots.append((sx, gx))
        lines += [f"{sx * 10.0:.3f} 10.000 {x * 10.0:.3f} 10.000" for x in gx]
    (tmp / "coords.txt").write_text("\n".join(lines) + "\n")
    (tmp / "CSG").mkdir(exist_ok=True)
    for is_, (sx, gx) in enumerate(shots):
        rng.standard_normal((len(gx), NT)).astype(np.float32).tofile(tmp / "CSG" / f"CSG{is_}.dat")
    wdir.mkdir(exist_ok=True)
    text = f"""ns {len(shots)}
ngmax {max(len(g) for _, g in shots)}
nx {NX}
nz {NZ}
nt {NT}
npml 10
delay {DELAY}
delaycal {DELAYCAL}
sbegin 0
send {len(shots) - 1}
dx 10.0
dz 10.0
dt 0.001
fr 25
velfx 0.0
planeTag 1
np 5
dp 0.0013
pmin -0.0031
precsg {tmp}/CSG/CSG
wdir {wdir}/
v0file {tmp}/v0.bin
coordfile {tmp}/coords.txt
"""
    path = tmp / f"param_{wdir.name}.txt"
    path.write_text(text)
    return path


def test_plane_prepare_matches_reference(tmp_path):
    rng = np.random.default_rng(2)
    param = write_survey(tmp_path, tmp_path / "OURS", rng)
    with Driver(None, str(param)) as d:
        d.plane_prepare()
        np_, pmin, dp = d.params.np, d.params.pmin, d.params.dp
    # the same steps from the reference's pieces
    ng, sc, gc = [], [], []
    lines = (tmp_path / "coords.txt").read_text().split("\n")
    shots = {}
    for ln in lines:
        if ln.strip():
            a = [np.float32(v) for v in ln.split()]
            shots.setdefault(float(a[0]), (a[0], a[1], []))[2].append((a[2], a[3]))
    srcs = list(shots.values())
    ref = O.RefInversion(np.array([(s[0], s[1]) for s in srcs], np.float32),
                         [np.array([g[0] for g in s[2]], np.float32) for s in srcs],
                         [np.array([g[1] for g in s[2]], np.float32) for s in srcs],
                         np.float32(10.0), np.float32(10.0), np.float32(1e-3), np.float32(25.0),
                         np.float32(0.0), NX, NZ, NT)
    NTT = NT + DELAYCAL
    wav = O.ricker(np.float32(1e-3), np.float32(25.0), DELAY + DELAYCAL, NTT, impl="ref")
    data = [np.fromfile(tmp_path / "CSG" / f"CSG{i}.dat", np.float32).reshape(len(s[2]), NT)
            for i, s in enumerate(srcs)]
    assert np_ == 5
    for k in range(np_):
        kx = np.float32(np.float32(pmin) + np.float32(k) * np.float32(dp))
        sou = np.zeros((NX, NTT), np.float32)
        rec = np.zeros((NX, NT), np.float32)
        for is_, s in enumerate(srcs):
            sx = np.float32(s[0])
            tw = O.ref_harmonic(wav, kx, sx)
            isx = int((sx - np.float32(0.0)) / np.float32(10.0) + np.float32(0.001))
            sou[isx] = sou[isx] + tw
            csgn = np.stack([O.ref_harmonic(tr, kx, sx) for tr in data[is_]])
            tr = np.zeros((NX, NT), np.float32)
            ref.swapreord(np.ascontiguousarray(csgn), is_, tr, np.float32(0.0), adj=False)
            rec = tr + rec
        got_s = np.fromfile(tmp_path / "OURS" / f"PLANE_S_NEW{k}.dat", np.float32).reshape(NX, NTT)
        got_r = np.fromfile(tmp_path / "OURS" / f"PLANE_R_NEW{k}.dat", np.float32).reshape(NX, NT)
        assert np.array_equal(got_s, sou), k
        assert np.array_equal(got_r, rec), k
        assert np.abs(got_r).max() > 0
    ref.close()


@pytest.mark.parametrize("half", [30, 100])
def test_hilbert_helper_matches_oracle(half):
    rng = np.random.default_rng(half)
    x = rng.standard_normal(517).astype(np.float32)
    out = np.zeros_like(x)
    assert lib().seis_fd_hilbert(x.ctypes.data, out.ctypes.data, len(x), half) == 0
    assert np.array_equal(out, O.hilbert(x, half=half))
