"""Every tile shape of the step kernels (include/seis_fd.h SEIS_TILE_*) gives
the same results: the exact build equals the restatement of the reference
bit for bit on golden and random grids whose last tiles are ragged for every
shape; the exact adjoint of every shape matches the FP64 oracle; the
autotuner keeps one of the shapes and reuses its choice per plan signature."""
import numpy as np
import pytest

import oracle as O
from helpers import golden_cases, rel_l2
from seis_b200 import Shot
from seis_b200._lib import (IN_DV, IN_GATHER, IN_VEL, IN_WAVELET, OP_BORN, OP_BORN_ADJOINT,
                            OP_MODELING, OP_RTM, OUT_GATHER, OUT_IMAGE, SNAP_BF16, TILE_SHAPES,
                            Lsrtm, Plan)

pytestmark = pytest.mark.gpu
SHAPES = sorted(TILE_SHAPES)
IDS = [f"{TILE_SHAPES[s][0]}x{TILE_SHAPES[s][1]}" for s in SHAPES]


def run(ctx, op, s, wav, vel, shape, dv=None, rec=None, exact=True, out=OUT_GATHER):
    with Plan(ctx, op, [s]) as p:
        p.set_tile_shape(shape)
        assert p.tile_shape == shape
        if op != OP_BORN_ADJOINT:
            p.set_exact(exact)
        p.set(0, IN_VEL, vel)
        p.set(0, IN_WAVELET, wav)
        if dv is not None:
            p.set(0, IN_DV, dv)
        if rec is not None:
            p.set(0, IN_GATHER, rec)
        p.run()
        return p.get(0, out)


def cases():
    gold = {g.name: g for g in golden_cases()}
    out = [(g.shot, g.vel, g.dv, g.wav) for g in (gold["ragged"], gold["pml1"], gold["thin"])]
    # padded grids 97 x 65, 65 x 34, 65 x 129 and 210 x 150: ragged last tiles
    # in x and z for every shape
    for nx, nz, pml in ((95, 63, 1), (61, 30, 2), (33, 97, 16), (170, 110, 20)):
        rng = np.random.default_rng(nx * nz + pml)
        s = Shot(nx=nx, nz=nz, pml=pml, nt=90, ndel=20, sx=nx // 3, sz=nz // 4, dt=1e-3,
                 dx=10.0, dz=12.0, gz=rng.integers(0, nz, nx))
        vel = (1500 + 2500 * rng.random((nx, nz))).astype(np.float32)
        dv = (rng.standard_normal((nx, nz)) * 50).astype(np.float32)
        out.append((s, vel, dv, O.ricker(s.dt, 25.0, s.ndel, s.NT)))
    return out


@pytest.mark.parametrize("shape", SHAPES, ids=IDS)
def test_exact_build_matches_restatement(ctx, shape):
    for s, vel, dv, wav in cases():
        rec = O.modeling(s, wav, vel)
        assert np.array_equal(run(ctx, OP_MODELING, s, wav, vel, shape), rec)
        assert np.array_equal(run(ctx, OP_BORN, s, wav, vel, shape, dv=dv), O.born(s, wav, vel, dv))
        img = run(ctx, OP_RTM, s, wav, vel, shape, rec=rec, out=OUT_IMAGE)
        assert np.array_equal(img, O.rtm(s, wav, vel, rec))


@pytest.mark.parametrize("shape", SHAPES, ids=IDS)
def test_fast_build_and_adjoint(ctx, shape):
    for s, vel, dv, wav in cases()[3:]:
        exact = O.born(s, wav, vel, dv)
        fast = run(ctx, OP_BORN, s, wav, vel, shape, dv=dv, exact=False)
        assert rel_l2(fast, exact) <= 1e-5
        d = np.random.default_rng(s.nx).standard_normal((s.nx, s.nt)).astype(np.float32)
        img = run(ctx, OP_BORN_ADJOINT, s, wav, vel, shape, rec=d, out=OUT_IMAGE)
        ref = O.born_adjoint(s, wav.astype(np.float64), vel, d, prec="f64")
        assert rel_l2(img, ref) < 2e-5


def test_autotune_keeps_a_shape_and_caches_it(ctx):
    s, vel, dv, wav = cases()[-1]
    with Plan(ctx, OP_BORN, [s]) as p:
        p.set(0, IN_VEL, vel)
        p.set(0, IN_WAVELET, wav)
        p.set(0, IN_DV, dv)
        best, ms = p.autotune(steps=5, force=True)
        assert best in SHAPES and p.tile_shape == best
        assert all(t > 0 for t in ms) and ms[best] == min(ms)
        p.run()
        assert np.array_equal(p.get(0, OUT_GATHER), O.born(s, wav, vel, dv))
    with Plan(ctx, OP_BORN, [s]) as q:  # same signature: the cached choice, untimed
        q.set(0, IN_VEL, vel)
        q.set(0, IN_WAVELET, wav)
        best2, ms2 = q.autotune(steps=5)
        assert best2 == best and q.tile_shape == best and not any(ms2)


def test_lsrtm_shapes_agree(ctx):
    """The solver with a fixed shape and with the autotuner's choice follows
    the same iterates to FP32 rounding (the adjoint's one-cell halo of ring
    terms is formed per tile, so tile borders differ in rounding only)."""
    s, vel, dv, wav = cases()[-1]
    d = O.born(s, wav, vel, dv)
    out = []
    for shape in (None, SHAPES[0], SHAPES[2], SHAPES[4]):
        with Lsrtm(ctx, s.nx, s.nz, [s], [0], snap_every=2, snap_dtype=SNAP_BF16,
                   tile_shape=shape) as ls:
            ls.set_background(vel, wav)
            ls.set_data(0, d)
            h = [ls.reset()] + list(ls.iterate(2))
            out.append((np.array(h), ls.model()))
    for h, m in out[1:]:
        assert np.max(np.abs(h - out[0][0]) / out[0][0]) <= 1e-5
        assert rel_l2(m, out[0][1]) <= 1e-5


@pytest.mark.parametrize("flags", [0, 1, 2, 3, 4, 5], ids=lambda f: f"launch{f}")
def test_launch_forms_agree(ctx, flags):
    """Every launch form -- the interior and pad kernels one after the other
    or overlapped, the interior kernel persistent (forced even for a few
    tiles) or one tile per CTA -- gives the reference's results bit for bit,
    and the exact adjoint the same image in every form."""
    from seis_b200._lib import LAUNCH_OVERLAP, LAUNCH_PERSISTENT, LAUNCH_PER_TILE  # noqa: F401
    s, vel, dv, wav = cases()[-1]
    for op, kw, ref in ((OP_MODELING, {}, O.modeling(s, wav, vel)),
                        (OP_BORN, {"dv": dv}, O.born(s, wav, vel, dv))):
        with Plan(ctx, op, [s, s]) as p:
            p.set_launch(flags)
            assert p.launch == flags
            for i in range(2):
                p.set(i, IN_VEL, vel)
                p.set(i, IN_WAVELET, wav)
                if "dv" in kw:
                    p.set(i, IN_DV, kw["dv"])
            p.run()
            for i in range(2):
                assert np.array_equal(p.get(i, OUT_GATHER), ref)
    d = np.random.default_rng(3).standard_normal((s.nx, s.nt)).astype(np.float32)
    imgs = []
    for f in (0, flags):
        with Plan(ctx, OP_BORN_ADJOINT, [s]) as p:
            p.set_launch(f)
            p.set(0, IN_VEL, vel)
            p.set(0, IN_WAVELET, wav)
            p.set(0, IN_GATHER, d)
            p.run()
            imgs.append(p.get(0, OUT_IMAGE))
    assert np.array_equal(imgs[0], imgs[1])
