"""The oracle CGLS (FP64): the data residual decreases at every iteration."""
import numpy as np

import oracle as O
from seis_b200 import Shot


def test_oracle_cgls_reduces_residual():
    nx, nz, nsx, nt = 40, 30, 28, 140
    x0 = [0, 12]
    shots = [Shot(nx=nsx, nz=nz, pml=6, nt=nt, ndel=20, sx=nsx // 2, sz=2, dt=1e-3, dx=10.0,
                  dz=10.0, gz=np.full(nsx, 1)) for _ in x0]
    v0 = np.full((nx, nz), 2000.0, np.float32)
    m_true = np.zeros((nx, nz), np.float32)
    m_true[:, 18] = 100.0
    wav = O.ricker(1e-3, 25.0, 20, nt + 20)
    dobs = [O.born(s, wav, v0[x:x + s.nx], m_true[x:x + s.nx], prec="f64") for s, x in zip(shots, x0)]
    m, rr0, hist = O.lsrtm_cgls(nx, nz, shots, x0, wav, v0, dobs, 5)
    assert np.all(np.diff([rr0] + hist) < 0)
    assert hist[-1] < 0.7 * rr0
