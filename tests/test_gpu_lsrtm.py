"""LSRTM by CGLS on the GPU against the FP64 oracle CGLS (same operators,
same global model, shots on overlapping apertures)."""
import numpy as np
import pytest

import oracle as O
from helpers import rel_l2
from seis_b200 import Shot
from seis_b200._lib import SNAP_BF16, SNAP_F16, SNAP_F32, Lsrtm

pytestmark = pytest.mark.gpu


def survey(nx=96, nz=60, nsx=48, nshot=3, pml=12, nt=260, seed=4):
    rng = np.random.default_rng(seed)
    x0 = [int(round(k * (nx - nsx) / max(nshot - 1, 1))) for k in range(nshot)]
    shots = [Shot(nx=nsx, nz=nz, pml=pml, nt=nt, ndel=25, sx=nsx // 2, sz=2, dt=1e-3, dx=10.0,
                  dz=10.0, gz=np.full(nsx, 1)) for _ in range(nshot)]
    z = np.arange(nz)
    v0 = np.broadcast_to(1900.0 + 12.0 * z, (nx, nz)).astype(np.float32).copy()
    m_true = np.zeros((nx, nz), np.float32)
    m_true[:, nz // 2] = 150.0
    m_true[nx // 3:nx // 3 + 10, nz // 3] = -100.0
    wav = O.ricker(1e-3, 25.0, 25, nt + 25)
    dobs = [O.born(s, wav, v0[x:x + s.nx], m_true[x:x + s.nx]) for s, x in zip(shots, x0)]
    return nx, nz, shots, x0, wav, v0, m_true, dobs


def run_gpu(ctx, sv, niter, **kw):
    nx, nz, shots, x0, wav, v0, _, dobs = sv
    with Lsrtm(ctx, nx, nz, shots, x0, **kw) as ls:
        ls.set_background(v0, wav)
        for k, d in enumerate(dobs):
            ls.set_data(k, d)
        rr0 = ls.reset()
        hist = ls.iterate(niter)
        return ls.model(), rr0, hist


def test_lsrtm_matches_fp64_cgls(ctx):
    sv = survey()
    nx, nz, shots, x0, wav, v0, _, dobs = sv
    niter = 4
    m_ref, rr0_ref, hist_ref = O.lsrtm_cgls(nx, nz, shots, x0, wav, v0, dobs, niter)
    m, rr0, hist = run_gpu(ctx, sv, niter, snap_dtype=SNAP_F32, exact=True)
    print("rr0", rr0, rr0_ref)
    print("gpu ", hist / rr0)
    print("fp64", np.array(hist_ref) / rr0_ref)
    assert abs(rr0 - rr0_ref) <= 1e-6 * rr0_ref
    assert np.all(np.diff(hist) < 0) and hist[0] < rr0
    np.testing.assert_allclose(hist / rr0, np.array(hist_ref) / rr0_ref, rtol=2e-3, atol=1e-5)
    err = rel_l2(m, m_ref)
    print("model rel L2 vs FP64 CGLS", err)
    assert err < 2e-3


def test_lsrtm_bf16_snapshots_and_repeat(ctx):
    """The default configuration (BF16 snapshots, fast kernels) follows the FP64
    solver closely, and a reset reproduces the same iterates bit for bit."""
    sv = survey(seed=5)
    nx, nz, shots, x0, wav, v0, _, dobs = sv
    niter = 3
    m_ref, rr0_ref, hist_ref = O.lsrtm_cgls(nx, nz, shots, x0, wav, v0, dobs, niter)
    nx, nz, shots, x0, wav, v0, _, dobs = sv
    with Lsrtm(ctx, nx, nz, shots, x0, snap_dtype=SNAP_BF16) as ls:
        ls.set_background(v0, wav)
        for k, d in enumerate(dobs):
            ls.set_data(k, d)
        rr0 = ls.reset()
        h1 = ls.iterate(niter)
        m1 = ls.model()
        ls.reset()
        h2 = ls.iterate(niter)
        m2 = ls.model()
    assert np.array_equal(h1, h2) and np.array_equal(m1, m2)
    np.testing.assert_allclose(h1 / rr0, np.array(hist_ref) / rr0_ref, rtol=2e-2, atol=1e-4)
    assert rel_l2(m1, m_ref) < 2e-2


def test_vector_ops_match_opern(ctx):
    """seis_fd_vec_dot / seis_fd_vec_axpby follow DOTPRODUCT (FP32 product,
    FP64 sum) and ADDSCAL (formed in double) of src/util/arraymath.h."""
    import torch
    from seis_b200._lib import vec_axpby, vec_dot
    rng = np.random.default_rng(1)
    for n in (1, 1000, 3_000_001):
        a = rng.standard_normal(n).astype(np.float32)
        b = rng.standard_normal(n).astype(np.float32)
        ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        torch.cuda.synchronize()
        got = vec_dot(ctx, ta.data_ptr(), tb.data_ptr(), n)
        want = float(np.sum((a * b).astype(np.float64)))
        assert abs(got - want) <= 1e-12 * np.sum(np.abs(a * b).astype(np.float64))
        vec_axpby(ctx, tb.data_ptr(), ta.data_ptr(), 0.3, -1.7, n)
        want_y = (0.3 * a.astype(np.float64) - 1.7 * b.astype(np.float64)).astype(np.float32)
        assert np.array_equal(tb.cpu().numpy(), want_y)


def test_phase_loop_reproduces_iterate(ctx):
    """The sharded CG loop on one device (nothing to sum) gives the same
    iterates as seis_fd_lsrtm_iterate, bit for bit."""
    from seis_b200.shards import DeviceEngine, ShardedCGLS
    sv = survey(seed=6)
    nx, nz, shots, x0, wav, v0, _, dobs = sv
    with Lsrtm(ctx, nx, nz, shots, x0) as ls:
        ls.set_background(v0, wav)
        for k, d in enumerate(dobs):
            ls.set_data(k, d)
        rr0 = ls.reset()
        h1 = ls.iterate(3)
        m1 = ls.model()
        cg = ShardedCGLS(DeviceEngine(ls), lambda b: None)
        rr0b = cg.reset()
        h2 = cg.iterate(3)
        m2 = ls.model()
    assert rr0 == rr0b
    assert np.array_equal(h1, np.array(h2)) and np.array_equal(m1, m2)


def test_lsrtm_with_checkpoints_is_bit_identical(ctx):
    """CGLS with source-field checkpoints every 20 steps (snapshots every 4
    steps recomputed per segment) reproduces the solver that keeps every
    snapshot, model and residual history bit for bit."""
    sv = survey()
    m0, rr0, h0 = run_gpu(ctx, sv, 3, snap_every=4)
    m1, rr1, h1 = run_gpu(ctx, sv, 3, snap_every=4, checkpoint_every=20)
    assert rr0 == rr1
    assert np.array_equal(h0, h1)
    assert np.array_equal(m0, m1)


@pytest.mark.parametrize("group,ck", [(1, 0), (2, 20)])
def test_lsrtm_in_shot_groups_is_bit_identical(ctx, group, ck):
    """CGLS that builds the plans of `group` shots at a time in every operator
    application (for surveys whose plans do not fit on the device at once),
    with or without checkpoints, reproduces the solver that keeps every plan,
    model and residual history bit for bit.  The tile shape is fixed: the
    autotuner may pick another shape for a group's plans than for the whole
    survey's, and the exact adjoint's ring terms on tile borders then differ
    in rounding."""
    from seis_b200._lib import TILE_32x64
    sv = survey()
    m0, rr0, h0 = run_gpu(ctx, sv, 3, snap_every=4, tile_shape=TILE_32x64)
    m1, rr1, h1 = run_gpu(ctx, sv, 3, snap_every=4, checkpoint_every=ck, group_shots=group,
                          tile_shape=TILE_32x64)
    assert rr0 == rr1
    assert np.array_equal(h0, h1)
    assert np.array_equal(m0, m1)


@pytest.mark.parametrize("name,kw,tol", [
    ("f16_every4_fast", dict(snap_every=4, snap_dtype=SNAP_F16), 1e-3),
    ("f16_every4_fast_checkpoints", dict(snap_every=4, snap_dtype=SNAP_F16, checkpoint_every=64),
     1e-3),
    ("f32_every1_exact", dict(snap_every=1, snap_dtype=SNAP_F32, exact=True), 1e-3),
    ("bf16_every4_fast", dict(snap_every=4, snap_dtype=SNAP_BF16), 2e-3),
])
def test_lsrtm_1200x400_subset_vs_fp64_cgls(ctx, name, kw, tol):
    """Two shots of the 1200 x 400 LSRTM survey (nt cut to 500), three CG
    iterations, against the FP64 CGLS of the same shots and data
    (tests/golden/lsrtm_fp64.npz, made by tests/golden/make_lsrtm_fp64.py):
    the residual curve and the model (on the fixture's every-4th-cell
    subsample) within 1e-3 relative -- the solver's default FP16 snapshots
    and FP32 ones.  BF16 snapshots (7 mantissa bits) follow the residual
    curve to 8e-5 but the model only to 1.6e-3, gated at 2e-3."""
    import hashlib
    import os

    from helpers import GOLDEN
    from seis_b200 import synth
    g = np.load(os.path.join(GOLDEN, "lsrtm_fp64.npz"))
    sv = synth.lsrtm(nt=int(g["nt"])).subset([int(k) for k in g["shots"]])
    wav = sv.wavelet()
    dobs = [O.born(s, wav.astype(np.float64), sv.sub(sv.vel0, i), sv.sub(sv.dv, i),
                   prec="f64").astype(np.float32) for i, s in enumerate(sv.shots)]
    assert [hashlib.sha256(d.tobytes()).hexdigest() for d in dobs] == [str(h) for h in g["data_sha"]]
    with Lsrtm(ctx, sv.nx, sv.nz, sv.shots, sv.x0, **kw) as ls:
        ls.set_background(sv.vel0, wav)
        for k, d in enumerate(dobs):
            ls.set_data(k, d)
        rr0 = ls.reset()
        hist = ls.iterate(int(g["niter"]))
        m = ls.model()
    st = int(g["step"])
    err_m = rel_l2(m[::st, ::st], g["m_sub"])
    ref_h = g["hist"] / g["rr0"]
    err_h = float(np.max(np.abs(hist / rr0 - ref_h) / ref_h))
    print(f"{name}: rr0 rel {abs(rr0 - g['rr0']) / g['rr0']:.2e}, residual curve rel "
          f"{err_h:.2e}, model rel L2 {err_m:.2e} vs FP64 CGLS")
    assert abs(rr0 - float(g["rr0"])) <= 1e-6 * float(g["rr0"])
    assert err_h <= 1e-3 and err_m <= tol
