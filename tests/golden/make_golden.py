"""Generate the golden fixtures in tests/golden/*.npz by running the
reference's own FD code (src/util/fd.cpp, compiled unmodified into
oracle/_ref/libseisref.so by oracle/Makefile).

The reference ships no tests, fixtures or golden vectors, so these files are
the pin for both the C restatement (oracle/) and the CUDA path.  Inputs are
small seeded synthetic models; every case is stored with its inputs.

Run from the repository root after `make -C oracle`:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


class Case:
    def __init__(self, name, nx, nz, pml, nt, ndel, sx, sz, dt, dx, dz, fr, gz, vel, dv):
        self.name, self.nx, self.nz, self.pml = name, nx, nz, pml
        self.nt, self.ndel, self.sx, self.sz = nt, ndel, sx, sz
        self.dt, self.dx, self.dz, self.fr = dt, dx, dz, fr
        self.gz = np.ascontiguousarray(gz, np.int32)
        self.vel = np.ascontiguousarray(vel, np.float32)
        self.dv = np.ascontiguousarray(dv, np.float32)


def smooth_random(rng, nx, nz, lo, hi, k=5):
    a = rng.random((nx + k, nz + k))
    c = np.cumsum(np.cumsum(a, 0), 1)
    box = c[k:, k:] - c[:-k, k:] - c[k:, :-k] + c[:-k, :-k]
    box = (box - box.min()) / (box.max() - box.min() + 1e-12)
    return (lo + (hi - lo) * box[:nx, :nz]).astype(np.float32)


def cases():
    out = []
    rng = np.random.default_rng(1234)
    # ragged receiver depths, dx != dz, source on the top interior row
    nx, nz = 57, 43
    out.append(Case("ragged", nx, nz, 10, 250, 40, 20, 0, 1e-3, 10.0, 12.5, 15.0,
                    rng.integers(0, 4, nx), smooth_random(rng, nx, nz, 2000, 3500),
                    rng.standard_normal((nx, nz)) * 100))
    # thinnest pad, source and receivers next to the pad
    nx, nz = 30, 20
    out.append(Case("pml1", nx, nz, 1, 120, 20, 0, 0, 1e-3, 10.0, 10.0, 20.0,
                    np.zeros(nx), smooth_random(rng, nx, nz, 1800, 2600),
                    rng.standard_normal((nx, nz)) * 50))
    # thin model: boundary strips of top and bottom overlap (nz < 8)
    nx, nz = 40, 5
    out.append(Case("thin", nx, nz, 6, 100, 15, 33, 2, 1e-3, 10.0, 10.0, 25.0,
                    np.full(nx, 4), smooth_random(rng, nx, nz, 2000, 2200),
                    rng.standard_normal((nx, nz)) * 20))
    # the 201x201 gradient-over-reflector model at half scale
    nx = nz = 101
    z = np.arange(nz) * 20.0
    vel = np.tile(np.where(z < 1000.0, 2000.0 + 0.5 * z, 3000.0), (nx, 1))
    out.append(Case("gradient", nx, nz, 20, 400, 100, 50, 1, 1e-3, 20.0, 20.0, 15.0,
                    np.full(nx, 1), vel, np.where(np.abs(z - 400.0) < 60, 200.0, 0.0) * np.ones((nx, 1))))
    # layered model, coarse
    nx, nz = 96, 48
    vals = np.sort(rng.uniform(1500, 4500, 8))
    vel = np.repeat(vals, nz // 8)[None, :].repeat(nx, 0)
    out.append(Case("layered", nx, nz, 12, 300, 50, 47, 1, 1e-3, 12.5, 12.5, 20.0,
                    np.ones(nx), vel, vel - vel.mean()))
    return out


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libseisref.so is missing: run make -C oracle")
    O.ref_set_threads(1)
    for c in cases():
        NT = c.nt + c.ndel
        wav = O.ricker(c.dt, c.fr, c.ndel, NT, impl="ref")
        rec = O.modeling(c, wav, c.vel, impl="ref")
        born = O.born(c, wav, c.vel, c.dv, impl="ref")
        img = O.rtm(c, wav, c.vel, rec, impl="ref")
        x = np.random.default_rng(7).standard_normal(173).astype(np.float32)
        np.savez_compressed(
            os.path.join(OUT, f"{c.name}.npz"),
            scalars=np.array([c.nx, c.nz, c.pml, c.nt, c.ndel, c.sx, c.sz], np.int32),
            fscalars=np.array([c.dt, c.dx, c.dz, c.fr], np.float32),
            gz=c.gz, vel=c.vel, dv=c.dv, wav=wav, rec=rec, born=born, img=img,
            abs=O.set_abs(c.nz, c.nx, c.pml, impl="ref"),
            velpml=O.set_vel(c.vel, c.pml, impl="ref"),
            hil_in=x, hil_out=O.hilbert(x, impl="ref"))
        print(c.name, "rec", float(np.abs(rec).max()), "born", float(np.abs(born).max()),
              "img", float(np.abs(img).max()))


if __name__ == "__main__":
    main()
