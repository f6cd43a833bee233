"""Shared helpers of the test suite: golden fixtures and error metrics."""
import glob
import os

import numpy as np

from seis_b200 import Shot

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class Golden:
    def __init__(self, path):
        d = np.load(path)
        self.name = os.path.splitext(os.path.basename(path))[0]
        nx, nz, pml, nt, ndel, sx, sz = (int(v) for v in d["scalars"])
        dt, dx, dz, fr = (float(v) for v in d["fscalars"])
        self.shot = Shot(nx=nx, nz=nz, pml=pml, nt=nt, ndel=ndel, sx=sx, sz=sz, dt=dt, dx=dx,
                         dz=dz, gz=d["gz"])
        self.fr = fr
        for k in ("vel", "dv", "wav", "rec", "born", "img", "abs", "velpml", "hil_in", "hil_out"):
            setattr(self, k, d[k])


def _case_files():
    """The single-shot case fixtures (make_golden.py); the other archives in
    tests/golden hold benchmark-size results of their own layout."""
    out = []
    for p in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        with np.load(p) as d:
            if "scalars" in d.files:
                out.append(p)
    return out


def golden_cases():
    return [Golden(p) for p in _case_files()]


def golden_ids():
    return [os.path.splitext(os.path.basename(p))[0] for p in _case_files()]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def fd_args(s):
    """Positional scalar arguments of the reference call surface (fd.h:3)."""
    return (s.dt, s.dx, s.dz, s.nt, s.ndel, s.nx, s.nz, s.pml, s.sx, s.sz, s.gz)
