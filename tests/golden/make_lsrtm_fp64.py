"""Generate tests/golden/lsrtm_fp64.npz: FP64 CGLS on a subset of the
1200 x 400 LSRTM survey, for the GPU solver's configurations
(tests/test_gpu_lsrtm.py).

Survey: seis_b200.synth.lsrtm (1200 x 400 cells at 10 m, pml 40, layered
model with three dipping faults, dt 0.8 ms, 20 Hz), shots 8 and 24 of its 32
(full-aperture receivers at row 1), the time axis cut to nt = 500 (+ 94 delay
steps) to keep the FP64 run to minutes.  Observed data: FP64 Born modeling of
the true perturbation, rounded to float32.  Solver: the restatement's FP64
CGLS (oracle.lsrtm_cgls: FP64 Born operator and its exact transpose), three
iterations from a zero model.

Stored: the observed data's SHA-256, |d|^2, the residual after each
iteration, the model's L2 norm and the model on every 4th column and row.
From the repository root after `make -C oracle` (about 5 minutes):
    python tests/golden/make_lsrtm_fp64.py
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402
from seis_b200 import synth  # noqa: E402  (numpy-only survey module)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lsrtm_fp64.npz")
SHOTS, NT, NITER, STEP = (8, 24), 500, 3, 4


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def main():
    sv = synth.lsrtm(nt=NT).subset(SHOTS)
    wav = O.ricker(sv.dt, sv.fr, sv.ndel, sv.nt + sv.ndel)
    t = time.time()
    dobs = [O.born(s, wav.astype(np.float64), sv.sub(sv.vel0, i), sv.sub(sv.dv, i),
                   prec="f64").astype(np.float32) for i, s in enumerate(sv.shots)]
    print(f"FP64 Born data {time.time() - t:.0f} s", flush=True)
    t = time.time()
    m, rr0, hist = O.lsrtm_cgls(sv.nx, sv.nz, sv.shots, sv.x0, wav, sv.vel0, dobs, NITER)
    print(f"FP64 CGLS {time.time() - t:.0f} s: rr0 {rr0:.6e} hist {hist}", flush=True)
    np.savez_compressed(OUT, shots=np.array(SHOTS, np.int32), nt=np.int32(NT),
                        niter=np.int32(NITER), step=np.int32(STEP),
                        data_sha=np.array([sha(d) for d in dobs]),
                        rr0=np.float64(rr0), hist=np.array(hist, np.float64),
                        m_norm=np.linalg.norm(m), m_sub=np.asarray(m[::STEP, ::STEP], np.float32))
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
