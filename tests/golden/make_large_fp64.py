"""Generate tests/golden/large_fp64.npz: the FP64 image of one shot of the
largest benchmark survey, against which the benchmark and the GPU tests state
the image error of the mixed-storage and plain FP32 adjoints.

Survey: 4000 x 1000 cells at 5 m, nt 8000 + 120 delay, dt 0.5 ms, 25 Hz,
layered model with anomalies (seis_b200.synth.large_sweep, velocities capped
at 3000 m/s).  Shot 64 of its 256 (aperture 1137 columns starting at column
2399).  Observed data: the reference's own Born modeling of the true
perturbation over the smooth background (src/util/fd.cpp:81-177, compiled
into oracle/_ref), which the CUDA exact build reproduces bit for bit.  Image:
the exact Born adjoint of that gather, every step (source terms recomputed
from checkpoints every 256 steps: the same image), in the C restatement's
double build (oracle/seis_oracle_body.h, FP64 throughout).

Stored: the SHA-256 of the float32 inputs, the image's L2 norm, and the image
on every 4th column and every 4th row (float32).  Runs about 15 minutes on 8
cores; from the repository root after `make -C oracle`:
    python tests/golden/make_large_fp64.py
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

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "large_fp64.npz")
SHOT, STEP = 64, 4


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libseisref.so is missing: run make -C oracle REF=...")
    O.ref_set_threads(os.cpu_count() or 1)
    sv = synth.large_sweep(vmax=3000.0)
    s = sv.shots[SHOT]
    vel0, dv = sv.sub(sv.vel0, SHOT), sv.sub(sv.dv, SHOT)
    wav = O.ricker(s.dt, sv.fr, s.ndel, s.NT, impl="ref")
    t = time.time()
    d = O.born(s, wav, vel0, dv, impl="ref")
    print(f"Born data {time.time() - t:.0f} s, max|d| {np.abs(d).max():.4g}", flush=True)
    t = time.time()
    img = O.born_adjoint_ck(s, wav.astype(np.float64), vel0, d, 256, prec="f64")
    print(f"FP64 adjoint {time.time() - t:.0f} s, max|img| {np.abs(img).max():.4g}", flush=True)
    np.savez_compressed(OUT, shot=np.int32(SHOT), step=np.int32(STEP),
                        vel0_sha=sha(vel0), dv_sha=sha(dv), wav_sha=sha(wav), data_sha=sha(d),
                        img_norm=np.linalg.norm(img),
                        img_sub=np.asarray(img[::STEP, ::STEP], np.float32))
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
