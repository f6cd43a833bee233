"""CUDA path against the reference, on the GPU.

Bar: the kernels evaluate every cell in the reference's operation order with
no contraction, so gathers and images must equal the reference's values
exactly (np.array_equal, which treats +0 and -0 as equal)."""
import numpy as np
import pytest

import oracle as O
from helpers import fd_args, golden_cases, golden_ids, rel_l2
from seis_b200 import fd

pytestmark = pytest.mark.gpu
CASES = golden_cases()


@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_modeling_golden(ctx, g):
    rec = fd.modeling(*fd_args(g.shot), g.wav, g.vel, ctx=ctx)
    assert np.array_equal(rec, g.rec), rel_l2(rec, g.rec)


@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_born_golden(ctx, g):
    rec = fd.forward(*fd_args(g.shot), g.wav, g.vel, g.dv, ctx=ctx)
    assert np.array_equal(rec, g.born), rel_l2(rec, g.born)


@pytest.mark.parametrize("g", CASES, ids=golden_ids())
def test_rtm_golden(ctx, g):
    img = fd.adjoint(*fd_args(g.shot), g.wav, g.vel, g.rec, ctx=ctx)
    assert np.array_equal(img, g.img), rel_l2(img, g.img)


@pytest.mark.parametrize("seed", [5, 6, 7])
def test_random_cases_against_restatement(ctx, seed):
    from seis_b200 import Shot
    rng = np.random.default_rng(seed)
    nx, nz = int(rng.integers(20, 140)), int(rng.integers(8, 90))
    pml = int(rng.integers(1, 24))
    s = Shot(nx=nx, nz=nz, pml=pml, nt=int(rng.integers(40, 160)), ndel=int(rng.integers(0, 30)),
             sx=int(rng.integers(0, nx)), sz=int(rng.integers(0, nz)), dt=1e-3,
             dx=float(rng.uniform(8, 15)), dz=float(rng.uniform(8, 15)),
             gz=rng.integers(0, nz, nx))
    vel = (1500 + 2500 * rng.random((nx, nz))).astype(np.float32)
    dv = (rng.standard_normal((nx, nz)) * 50).astype(np.float32)
    wav = O.ricker(s.dt, 25.0, s.ndel, s.NT)
    rec = O.modeling(s, wav, vel)
    assert np.array_equal(fd.modeling(*fd_args(s), wav, vel, ctx=ctx), rec)
    assert np.array_equal(fd.forward(*fd_args(s), wav, vel, dv, ctx=ctx), O.born(s, wav, vel, dv))
    assert np.array_equal(fd.adjoint(*fd_args(s), wav, vel, rec, ctx=ctx), O.rtm(s, wav, vel, rec))


@pytest.mark.parametrize("nx,nz,pml", [(95, 63, 1), (61, 30, 2), (33, 97, 16)])
def test_tile_edge_sizes_against_restatement(ctx, nx, nz, pml):
    """Grids whose last tile column holds one or two columns (NX = 97, 65 = 1
    mod 32) or whose last tile row holds one row (NZ = 65, 129 = 1 mod 64):
    the frame's normal extrapolation then reaches cells of the previous tile."""
    from seis_b200 import Shot
    rng = np.random.default_rng(nx * nz + pml)
    s = Shot(nx=nx, nz=nz, pml=pml, nt=90, ndel=20, sx=nx // 3, sz=nz // 4, dt=1e-3, dx=10.0,
             dz=12.0, gz=rng.integers(0, nz, nx))
    vel = (1500 + 2500 * rng.random((nx, nz))).astype(np.float32)
    dv = (rng.standard_normal((nx, nz)) * 50).astype(np.float32)
    wav = O.ricker(s.dt, 25.0, s.ndel, s.NT)
    rec = O.modeling(s, wav, vel)
    assert np.array_equal(fd.modeling(*fd_args(s), wav, vel, ctx=ctx), rec)
    assert np.array_equal(fd.forward(*fd_args(s), wav, vel, dv, ctx=ctx), O.born(s, wav, vel, dv))
    assert np.array_equal(fd.adjoint(*fd_args(s), wav, vel, rec, ctx=ctx), O.rtm(s, wav, vel, rec))
