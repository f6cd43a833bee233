"""The exact-adjoint oracle (no reference counterpart) against the oracle's
Born operator: the dot-product test <L m, d> = <m, L^T d>."""
import numpy as np
import pytest

import oracle as O
from seis_b200 import Shot


@pytest.mark.parametrize("nx,nz,pml,dx,dz", [(40, 30, 8, 10.0, 12.5), (33, 9, 3, 10.0, 10.0),
                                             (50, 44, 1, 9.0, 11.0), (24, 20, 12, 10.0, 10.0)])
def test_dot_product_fp64(nx, nz, pml, dx, dz):
    rng = np.random.default_rng(nx * 100 + nz)
    s = Shot(nx=nx, nz=nz, pml=pml, nt=90, ndel=15, sx=nx // 2, sz=2, dt=1e-3, dx=dx, dz=dz,
             gz=rng.integers(0, nz, nx))
    vel = 1800 + 1500 * rng.random((nx, nz))
    wav = O.ricker(s.dt, 25.0, s.ndel, s.NT, prec="f64")
    m = rng.standard_normal((nx, nz))
    d = rng.standard_normal((nx, s.nt))
    a = float(np.sum(O.born(s, wav, vel, m, prec="f64") * d))
    b = float(np.sum(m * O.born_adjoint(s, wav, vel, d, prec="f64")))
    assert abs(a - b) <= 1e-12 * max(abs(a), abs(b))


@pytest.mark.parametrize("ck", [1, 7, 105, 500])
def test_checkpointed_adjoint_is_the_same_image(ck):
    """born_adjoint_ck (source terms recomputed per segment) equals
    born_adjoint (every source term kept) bit for bit, for segment lengths
    that divide the step count, do not, and exceed it."""
    rng = np.random.default_rng(ck)
    s = Shot(nx=37, nz=21, pml=6, nt=90, ndel=15, sx=12, sz=2, dt=1e-3, dx=10.0, dz=12.0,
             gz=rng.integers(0, 21, 37))
    vel = 1800 + 1500 * rng.random((37, 21))
    wav = O.ricker(s.dt, 25.0, s.ndel, s.NT, prec="f64")
    d = rng.standard_normal((37, s.nt))
    a = O.born_adjoint(s, wav, vel, d, prec="f64")
    b = O.born_adjoint_ck(s, wav, vel, d, ck, prec="f64")
    assert np.array_equal(a, b)
