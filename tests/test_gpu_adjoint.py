"""Exact Born adjoint on the GPU: against the FP64 oracle adjoint, and the
dot-product test against the GPU Born operator (FP32 gate: 1e-6 relative)."""
import numpy as np
import pytest

import oracle as O
from helpers import fd_args, rel_l2
from seis_b200 import Shot, fd
from seis_b200._lib import (IN_GATHER, IN_VEL, IN_WAVELET, OP_BORN_ADJOINT, OUT_IMAGE, SNAP_BF16,
                            SNAP_F16, SNAP_F32, Plan, SeisError)

pytestmark = pytest.mark.gpu

CASES = [(40, 30, 8, 10.0, 12.5), (33, 9, 3, 10.0, 10.0), (130, 100, 20, 10.0, 10.0),
         (200, 90, 40, 12.5, 12.5), (90, 150, 5, 9.0, 11.0)]


def make(nx, nz, pml, dx, dz, nt=160, seed=0):
    rng = np.random.default_rng(seed + nx * 7 + nz)
    s = Shot(nx=nx, nz=nz, pml=pml, nt=nt, ndel=20, sx=nx // 3, sz=3, dt=1e-3, dx=dx, dz=dz,
             gz=rng.integers(0, nz, nx))
    vel = (1800 + 1500 * rng.random((nx, nz))).astype(np.float32)
    wav = O.ricker(s.dt, 25.0, s.ndel, s.NT)
    m = rng.standard_normal((nx, nz)).astype(np.float32)
    d = rng.standard_normal((nx, nt)).astype(np.float32)
    return s, vel, wav, m, d


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}x{c[1]}p{c[2]}" for c in CASES])
def test_adjoint_matches_fp64_oracle(ctx, case):
    s, vel, wav, m, d = make(*case)
    img = fd.born_adjoint(*fd_args(s), wav, vel, d, ctx=ctx)
    ref = O.born_adjoint(s, wav.astype(np.float64), vel, d, prec="f64")
    err = rel_l2(img, ref)
    print(f"adjoint {case} vs FP64 oracle: rel L2 {err:.3e}")
    assert err < 2e-5


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}x{c[1]}p{c[2]}" for c in CASES])
def test_dot_product_fp32(ctx, case):
    s, vel, wav, m, d = make(*case, seed=3)
    Lm = fd.forward(*fd_args(s), wav, vel, m, ctx=ctx).astype(np.float64)
    Ltd = fd.born_adjoint(*fd_args(s), wav, vel, d, ctx=ctx).astype(np.float64)
    a, b = float(np.sum(Lm * d)), float(np.sum(m * Ltd))
    rel = abs(a - b) / max(abs(a), abs(b))
    # the same difference against the size of the terms: free of the
    # cancellation in <Lm, d> for random vectors
    rel_norm = abs(a - b) / (np.linalg.norm(Lm) * np.linalg.norm(d))
    print(f"dot test {case}: {a:.9e} {b:.9e} rel {rel:.3e} rel/|Lm||d| {rel_norm:.3e}")
    # FP32 recursions over ~200 steps: each operator carries ~5e-6 relative
    # rounding error (the transpose itself is exact: the FP64 oracle pair
    # passes at 1e-12)
    assert rel_norm <= 1e-6, (a, b)
    assert rel <= 1e-4, (a, b)


@pytest.mark.parametrize("every,dtype,tol", [(1, SNAP_BF16, 1e-3), (1, SNAP_F16, 2e-4),
                                             (2, SNAP_BF16, 1e-3), (4, SNAP_F32, 2e-4),
                                             (4, SNAP_BF16, 1e-3), (4, SNAP_F16, 3e-4)])
def test_mixed_snapshot_image_error(ctx, every, dtype, tol):
    """Snapshots thinned in time and/or stored in 16 bits: image error against
    the FP64 exact adjoint (all steps), for band-limited residuals (Born data
    of a random perturbation, as in an LSRTM iteration) and a wavelet delayed
    by 1.5 periods.  The GPU result is also held against the FP64 adjoint
    thinned the same way, which isolates the storage error from the thinning
    error."""
    s, vel, wav, m, _ = make(200, 90, 40, 12.5, 12.5, nt=300, seed=9)
    s = Shot(nx=s.nx, nz=s.nz, pml=s.pml, nt=s.nt, ndel=60, sx=s.sx, sz=s.sz, dt=s.dt, dx=s.dx,
             dz=s.dz, gz=s.gz)
    wav = O.ricker(s.dt, 25.0, s.ndel, s.NT)
    d = O.born(s, wav, vel, m)
    with Plan(ctx, OP_BORN_ADJOINT, [s]) as p:
        p.set_snapshots(every, dtype)
        p.set(0, IN_VEL, vel)
        p.set(0, IN_WAVELET, wav)
        p.set(0, IN_GATHER, d)
        p.run()
        img = p.get(0, OUT_IMAGE)
    w64 = wav.astype(np.float64)
    ref = O.born_adjoint(s, w64, vel, d, prec="f64")
    thin = ref if every == 1 else O.born_adjoint(s, w64, vel, d, prec="f64", every=every)
    err, err_thin, inherent = rel_l2(img, ref), rel_l2(img, thin), rel_l2(thin, ref)
    print(f"snapshots every {every} dtype {dtype}: image rel L2 {err:.3e} "
          f"(vs thinned FP64 {err_thin:.3e}; thinning alone {inherent:.3e})")
    assert err < tol
    assert err_thin < tol


def _adjoint_images(ctx, shots, vels, wav, gathers, every, dtype, ck, runs=2):
    """Images of a batch of shots from one adjoint plan, run `runs` times (the
    first run captures the graph, later runs replay it) with new gathers."""
    out = []
    with Plan(ctx, OP_BORN_ADJOINT, shots) as p:
        p.set_snapshots(every, dtype)
        if ck:
            p.set_checkpoints(ck)
        for i, v in enumerate(vels):
            p.set(i, IN_VEL, v)
            p.set(i, IN_WAVELET, wav)
        for r in range(runs):
            for i, d in enumerate(gathers):
                p.set(i, IN_GATHER, d * (1.0 + r))
            p.run()
            out.append([p.get(i, OUT_IMAGE) for i in range(len(shots))])
    return out


@pytest.mark.parametrize("every,dtype,ck", [(1, SNAP_F32, 7), (2, SNAP_BF16, 6),
                                            (4, SNAP_F16, 8), (4, SNAP_BF16, 64)])
def test_checkpointed_adjoint_is_bit_identical(ctx, every, dtype, ck):
    """Source-field checkpoints (the two time levels before every ck-th step,
    each segment's snapshots recomputed before the reverse steps that use them)
    give the same images, bit for bit, as keeping every snapshot: a ragged batch
    whose step count is not a multiple of ck, run twice through the graph."""
    rng = np.random.default_rng(31)
    shots, vels, gathers = [], [], []
    for nx, nz, pml in ((70, 44, 10), (41, 63, 3)):
        s = Shot(nx=nx, nz=nz, pml=pml, nt=181, ndel=25, sx=nx // 2, sz=2, dt=1e-3, dx=10.0,
                 dz=10.0, gz=rng.integers(0, nz, nx))
        shots.append(s)
        vels.append((1800 + 1500 * rng.random((nx, nz))).astype(np.float32))
        gathers.append(rng.standard_normal((nx, s.nt)).astype(np.float32))
    wav = O.ricker(1e-3, 25.0, 25, shots[0].NT)
    keep = _adjoint_images(ctx, shots, vels, wav, gathers, every, dtype, 0)
    ckpt = _adjoint_images(ctx, shots, vels, wav, gathers, every, dtype, ck)
    for r in range(2):
        for a, b in zip(keep[r], ckpt[r]):
            assert np.abs(a).max() > 0
            assert np.array_equal(a, b), (r, rel_l2(b, a))


def test_checkpoint_interval_must_hold_whole_snapshot_intervals(ctx):
    s, vel, wav, m, d = make(40, 30, 8, 10.0, 12.5)
    with Plan(ctx, OP_BORN_ADJOINT, [s]) as p:
        p.set_snapshots(4, SNAP_BF16)
        with pytest.raises(SeisError):
            p.set_checkpoints(6)
        p.set_checkpoints(8)
