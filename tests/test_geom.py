"""Per-shot geometry (include/seis_geom.h) against the reference's own
Inversion members, compiled from src/lsrtm/inversion.cpp into the oracle:
getVel, getIgz, swapReord, swapModel, removeDirect.  Index and copy work, so
the bar is bit-for-bit equality, over randomized surveys including apertures
that run past the model edges (clamped columns), off-grid receivers and the
reference's km-scale sample files (dx = 0.010)."""
import numpy as np
import pytest

import oracle as O
from seis_b200 import geom

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference oracle not built")


def survey(seed, dx, velfx, offgrid=False, nx=120, nz=50, ns=4):
    rng = np.random.default_rng(seed)
    dz = dx * (1.0 if seed % 2 else 1.25)
    x_lo, x_hi = velfx, velfx + (nx - 1) * dx
    sc, gxs, gzs = [], [], []
    for _ in range(ns):
        sx = np.float32(velfx + rng.integers(0, nx) * dx)
        sz = np.float32(rng.integers(0, 3) * dz)
        ng = int(rng.integers(10, 60))
        if offgrid:
            gx = rng.uniform(x_lo, x_hi, ng).astype(np.float32)
        else:
            g0 = int(rng.integers(0, nx - ng))
            gx = (velfx + (g0 + np.arange(ng)) * dx).astype(np.float32)
        gz = (rng.integers(0, 4, ng) * dz).astype(np.float32)
        sc.append((sx, sz))
        gxs.append(gx)
        gzs.append(gz)
    v = (1500 + 2000 * rng.random((nx, nz))).astype(np.float32)
    return dict(sc=np.array(sc, np.float32), gxs=gxs, gzs=gzs, dx=np.float32(dx),
                dz=np.float32(dz), velfx=np.float32(velfx), nx=nx, nz=nz, v=v, rng=rng)


CASES = [(1, 10.0, 0.0, False), (2, 12.5, 5.0, False), (3, 0.010, 0.0, False),
         (4, 10.0, 0.0, True), (5, 0.010, 0.25, True), (6, 7.5, 100.0, False)]
IDS = [f"seed{c[0]}-dx{c[1]}-fx{c[2]}{'-offgrid' if c[3] else ''}" for c in CASES]


def make_ref(s, nt, lpad, rpad, delay=10, dt=1e-3, fr=20.0):
    return O.RefInversion(s["sc"], s["gxs"], s["gzs"], s["dx"], s["dz"], dt, fr, s["velfx"],
                          s["nx"], s["nz"], nt, delay=delay, lpad=lpad, rpad=rpad)


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_aperture_and_subgrid_match_getvel(case):
    s = survey(*case)
    for lpad, rpad in ((0, 0), (20, 35), (200, 5)):
        ref = make_ref(s, 100, lpad, rpad)
        for is_ in range(len(s["gxs"])):
            fx, nxs, sub_ref = ref.getvel(is_, s["v"], float(s["velfx"]))
            fx2, nxs2 = geom.aperture(float(s["sc"][is_][0]), s["gxs"][is_], float(s["dx"]), lpad,
                                      rpad)
            assert (np.float32(fx2), nxs2) == (np.float32(fx), nxs)
            sub = geom.extract(s["v"], float(s["velfx"]), float(s["dx"]), fx2, nxs2)
            assert np.array_equal(sub, sub_ref)
        ref.close()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_receiver_rows_and_source_index(case):
    s = survey(*case)
    ref = make_ref(s, 100, 30, 30)
    for is_ in range(len(s["gxs"])):
        fx, nxs, _ = ref.getvel(is_, s["v"], float(s["velfx"]))
        igz_ref = ref.getigz(fx, nxs, is_)
        igz = geom.receiver_rows(s["gxs"][is_], s["gzs"][is_], fx, nxs, float(s["dx"]),
                                 float(s["dz"]), s["nz"])
        assert np.array_equal(igz, igz_ref)
        # source index as the worker loops form it (inversion.cpp:428-429)
        sx, sz = s["sc"][is_]
        want_x = int((np.float32(sx) - np.float32(fx)) / s["dx"] + np.float32(0.0001))
        want_z = int((np.float64(sz) - 0.0) / np.float64(s["dz"]) + np.float64(np.float32(1e-4)))
        assert geom.source_index(float(sx), float(sz), fx, float(s["dx"]), float(s["dz"])) == \
            (want_x, want_z)
    ref.close()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_trace_column_reorder_matches_swapreord(case):
    s = survey(*case)
    nt = 37
    ref = make_ref(s, nt, 15, 25)
    rng = s["rng"]
    for is_ in range(len(s["gxs"])):
        fx, nxs, _ = ref.getvel(is_, s["v"], float(s["velfx"]))
        ng = len(s["gxs"][is_])
        csg = rng.standard_normal((ng, nt)).astype(np.float32)
        rec_ref = rng.standard_normal((nxs, nt)).astype(np.float32)  # cleared by the call
        ref.swapreord(csg.copy(), is_, rec_ref, fx, adj=False)
        rec = geom.reorder_to_columns(csg, s["gxs"][is_], fx, nxs, float(s["dx"]))
        assert np.array_equal(rec, rec_ref)
        csg_ref = rng.standard_normal((ng, nt)).astype(np.float32)
        ref.swapreord(csg_ref, is_, rec.copy(), fx, adj=True)
        assert np.array_equal(geom.reorder_to_gather(rec, s["gxs"][is_], fx, float(s["dx"])),
                              csg_ref)
    ref.close()


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_image_scatter_matches_swapmodel(case):
    s = survey(*case)
    ref = make_ref(s, 10, 12, 40)
    rng = s["rng"]
    for is_ in range(len(s["gxs"])):
        fx, nxs, _ = ref.getvel(is_, s["v"], float(s["velfx"]))
        m = rng.standard_normal((nxs, s["nz"])).astype(np.float32)
        for add in (False, True):
            d0 = rng.standard_normal((s["nx"], s["nz"])).astype(np.float32)
            d_ref = d0.copy()
            ref.swapmodel(m.copy(), d_ref, fx, float(s["velfx"]), add)
            d = geom.swap_model(m, d0.copy(), fx, float(s["velfx"]), float(s["dx"]), add=add)
            assert np.array_equal(d, d_ref)
    ref.close()


@pytest.mark.parametrize("case", CASES, ids=IDS)
@pytest.mark.parametrize("delay", [0, 25])
def test_direct_arrival_mute_matches_removedirect(case, delay):
    s = survey(*case)
    nt = 900
    dt, fr = np.float32(5e-4 if s["dx"] > 1 else 1.6e-3), np.float32(25.0)
    v = s["v"] if s["dx"] > 1 else (s["v"] / 1000.0).astype(np.float32)  # km/s with km grids
    ref = make_ref(s, nt, 0, 0, delay=delay, dt=dt, fr=fr)
    rng = s["rng"]
    for is_ in range(len(s["gxs"])):
        ng = len(s["gxs"][is_])
        csg = rng.standard_normal((ng, nt)).astype(np.float32)
        want = csg.copy()
        ref.removedirect(want, v.copy(), is_)
        got = geom.remove_direct(csg.copy(), s["gxs"][is_], s["gzs"][is_], float(s["sc"][is_][0]),
                                 float(s["sc"][is_][1]), v, float(s["dx"]), float(s["dz"]),
                                 float(dt), float(fr), float(s["velfx"]), delay)
        assert np.array_equal(got, want)
        assert (got == 0).sum() > 0  # something was muted
    ref.close()
