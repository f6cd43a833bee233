"""The shot driver end to end on the GPU: parameter and coordinate files on
disk, modeling / Born / RTM gather and image files bit-for-bit against the
same pipeline composed from the reference's own compiled pieces (getVel,
getIgz, the operator, swapReord, removeDirect, swapModel), and LSRTM through
the driver against the FP64 CGLS with the same sub-grid column maps."""
import numpy as np
import pytest

import oracle as O
from helpers import rel_l2
from seis_b200 import Shot, geom
from seis_b200._lib import SNAP_F32
from seis_b200.driver import Driver

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_available(), reason="reference oracle not built")]

NX, NZ, DX, DZ, NT, DT, FR = 96, 40, 10.0, 10.0, 260, 1e-3, 25.0
DELAY, DELAYCAL, NPML, LPAD, RPAD = 5, 45, 10, 12, 9


def build_survey(tmp):
    rng = np.random.default_rng(11)
    z = np.arange(NZ)
    v = np.where(z < 22, 1800.0 + 10.0 * z, 2600.0).astype(np.float32)
    v = np.broadcast_to(v, (NX, NZ)).copy()
    v[40:55, 10:14] += 250.0
    from scipy.ndimage import gaussian_filter
    v0 = gaussian_filter(v, 3.0, mode="nearest").astype(np.float32)
    lines, shots = [], []
    for sx in (2, 30, 61, 93):  # the first and last apertures clamp at the model edges
        g0 = max(0, sx - 20)
        gx = np.arange(g0, min(NX, g0 + int(rng.integers(25, 40)))) * DX
        gz = np.full(gx.shape, 1 * DZ)
        shots.append((sx * DX, 1 * DZ, gx.astype(np.float32), gz.astype(np.float32)))
        lines += [f"{sx * DX:.3f} {DZ:.3f} {x:.3f} {zz:.3f}" for x, zz in zip(gx, gz)]
    (tmp / "CSG").mkdir()
    (tmp / "WDIR").mkdir()
    (tmp / "coords.txt").write_text("\n".join(lines) + "\n")
    v.tofile(tmp / "v.bin")
    v0.tofile(tmp / "v0.bin")
    ngmax = max(len(s[2]) for s in shots)
    (tmp / "param.txt").write_text(f"""! shot driver test survey
ns {len(shots)}
ngmax {ngmax}
nx {NX}
nz {NZ}
nt {NT}
npml {NPML}
delay {DELAY}
delaycal {DELAYCAL}
lpad {LPAD}
rpad {RPAD}
sbegin 0
send {len(shots) - 1}
dx {DX}
dz {DZ}
dt {DT}
fr {FR}
velfx 0.0
precsg {tmp}/CSG/CSG
wdir {tmp}/WDIR/
vfile {tmp}/v.bin
v0file {tmp}/v0.bin
coordfile {tmp}/coords.txt
""")
    return v, v0, shots


def reference(shots, v):
    sc = np.array([(s[0], s[1]) for s in shots], np.float32)
    return O.RefInversion(sc, [s[2] for s in shots], [s[3] for s in shots], DX, DZ, DT, FR, 0.0,
                          NX, NZ, NT, delay=DELAY, lpad=LPAD, rpad=RPAD)


def shot_of(ref, is_, shots, model):
    fx, nxs, sub = ref.getvel(is_, model, 0.0)
    igz = ref.getigz(fx, nxs, is_)
    sx, sz = shots[is_][0], shots[is_][1]
    isx = int((np.float32(sx) - np.float32(fx)) / np.float32(DX) + np.float32(1e-4))
    isz = int((np.float64(sz) - 0.0) / np.float64(np.float32(DZ)) + np.float64(np.float32(1e-4)))
    return fx, nxs, sub, Shot(nx=nxs, nz=NZ, pml=NPML, nt=NT, ndel=DELAYCAL, sx=isx, sz=isz,
                              dt=DT, dx=DX, dz=DZ, gz=igz)


@pytest.fixture(scope="module")
def survey(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("survey")
    v, v0, shots = build_survey(tmp)
    return tmp, v, v0, shots


def test_driver_modeling_born_rtm_match_reference_pipeline(ctx, survey):
    tmp, v, v0, shots = survey
    ref = reference(shots, v)
    wav = O.ricker(DT, FR, DELAY + DELAYCAL, NT + DELAYCAL, impl="ref")
    dv = (v - v0).astype(np.float32)
    with Driver(ctx, str(tmp / "param.txt"), batch=3) as d:
        d.modeling()
        d.born(dv)
        img = d.rtm(born_data=False)
    want_img = np.zeros((NX, NZ), np.float32)
    for is_, (sx, sz, gx, gz) in enumerate(shots):
        ng = len(gx)
        # modeling_MPI: getVel(v), modeling, swapReord(adj), removeDirect(v)
        fx, nxs, sub, shot = shot_of(ref, is_, shots, v)
        rec = O.modeling(shot, wav, sub, impl="ref")
        csg = np.zeros((ng, NT), np.float32)
        ref.swapreord(csg, is_, np.ascontiguousarray(rec), fx, adj=True)
        ref.removedirect(csg, v.copy(), is_)
        got = np.fromfile(tmp / "CSG" / f"CSG{is_}.dat", np.float32).reshape(ng, NT)
        assert np.array_equal(got, csg), f"shot {is_} gather"
        # forward_MPI: Born over getVel(v0), getVel(dv)
        fx0, nxs0, sub0, shot0 = shot_of(ref, is_, shots, v0)
        _, _, dsub = ref.getvel(is_, dv, 0.0)
        recb = O.born(shot0, wav, sub0, dsub, impl="ref")
        csgb = np.zeros((ng, NT), np.float32)
        ref.swapreord(csgb, is_, np.ascontiguousarray(recb), fx0, adj=True)
        ref.removedirect(csgb, v0.copy(), is_)
        gotb = np.fromfile(tmp / "WDIR" / f"BORN{is_}.dat", np.float32).reshape(ng, NT)
        assert np.array_equal(gotb, csgb), f"shot {is_} Born gather"
        # adjoint_MPI: removeDirect(v0), swapReord, RTM, swapModel, sum
        obs = csg.copy()
        ref.removedirect(obs, v0.copy(), is_)
        r = np.zeros((nxs0, NT), np.float32)
        ref.swapreord(obs, is_, r, fx0, adj=False)
        im = O.rtm(shot0, wav, sub0, r, impl="ref")
        tmpimg = np.zeros((NX, NZ), np.float32)
        ref.swapmodel(np.ascontiguousarray(im), tmpimg, fx0, 0.0, add=False)
        got_i = np.fromfile(tmp / "WDIR" / f"CSG_IMAGE{is_}.dat", np.float32).reshape(NX, NZ)
        assert np.array_equal(got_i, tmpimg), f"shot {is_} image"
        want_img = tmpimg + want_img
    assert np.array_equal(img, want_img)
    assert np.abs(img).max() > 0


def test_driver_lsrtm_matches_fp64_cgls(ctx, survey):
    tmp, v, v0, shots = survey
    niter = 3
    with Driver(ctx, str(tmp / "param.txt")) as d:
        d.born((v - v0).astype(np.float32))  # observed data: Born gathers
        m, rr = d.lsrtm(niter, born_data=True, snap_dtype=SNAP_F32, exact=True)
    # the same problem in FP64: apertures, column maps and observed columns
    ref = reference(shots, v)
    wav = O.ricker(DT, FR, DELAY + DELAYCAL, NT + DELAYCAL, impl="ref")
    descs, cols, dobs = [], [], []
    for is_, (sx, sz, gx, gz) in enumerate(shots):
        fx, nxs, sub, shot = shot_of(ref, is_, shots, v0)
        descs.append(shot)
        cols.append(geom.extract_columns(NX, 0.0, DX, fx, nxs))
        csg = np.fromfile(tmp / "WDIR" / f"BORN{is_}.dat", np.float32).reshape(len(gx), NT)
        ref.removedirect(csg, v0.copy(), is_)
        r = np.zeros((nxs, NT), np.float32)
        ref.swapreord(csg, is_, r, fx, adj=False)
        dobs.append(r)
    m_ref, rr0, hist = O.lsrtm_cgls(NX, NZ, descs, None, wav, v0, dobs, niter, cols=cols)
    print("rr gpu", rr / rr[0], "fp64", np.array([rr0] + hist) / rr0)
    assert abs(rr[0] - rr0) <= 1e-6 * rr0
    np.testing.assert_allclose(rr[1:] / rr[0], np.array(hist) / rr0, rtol=2e-3, atol=1e-5)
    err = rel_l2(m, m_ref)
    print("driver LSRTM model vs FP64 CGLS", err)
    assert err < 2e-3


def test_driver_illum_matches_reference_pipeline(ctx, survey):
    tmp, v, v0, shots = survey
    ref = reference(shots, v)
    wav = O.ricker(DT, FR, DELAY + DELAYCAL, NT + DELAYCAL, impl="ref")
    with Driver(ctx, str(tmp / "param.txt"), batch=2) as d:
        ss = d.illum()
    want = np.zeros((NX, NZ), np.float32)
    for is_ in range(len(shots)):
        fx, nxs, sub, shot = shot_of(ref, is_, shots, v0)
        sssub = O.illum(shot, wav, sub, impl="ref")
        tmpimg = np.zeros((NX, NZ), np.float32)
        ref.swapmodel(np.ascontiguousarray(sssub), tmpimg, fx, 0.0, add=False)
        got = np.fromfile(tmp / "WDIR" / f"ILLUM{is_}.dat", np.float32).reshape(NX, NZ)
        assert np.array_equal(got, tmpimg), f"shot {is_} illumination"
        want = tmpimg + want
    assert np.array_equal(ss, want)
