"""Generate tests/golden/configs.npz: the reference's own outputs at the full
sizes of the two single-shot benchmark configurations, for the GPU parity
tests (tests/test_gpu_configs.py).

* modeling, 201 x 201 at 10 m, gradient over a flat reflector, pml 40,
  nt 2000 + 100 delay, 15 Hz, source (100, 2), receivers at row 2
  (src/util/fd.cpp:15-80);
* Born modeling of the 20-layer 737 x 240 model's reflectivity over its
  Gaussian-smoothed background (sigma 10 cells), nt 4000 + 75, 20 Hz, source
  (368, 1), receivers at row 1 (fd.cpp:81-177), and the reference RTM of that
  Born gather (fd.cpp:592-719);
* the same modeling and Born gathers from the restatement's double build
  (FP64), to state every FP32 result's error against an FP64 run;
* the dot-product test of the FP64 Born operator and its exact transpose
  (the C restatement's double build) on the same 737 x 240 shot with seeded
  N(0, 1) vectors m (737 x 240, rng seed 22) and d (737 x 4000, drawn next).

Each output is stored as the SHA-256 of its float32 bytes (layout [nx][nt] or
[nx][nz], C order), its L2 norm and a regular subsample (every 16th trace of
the modeling gather, every 48th of the Born gather, every 8th column of the
image), with the SHA-256 of the inputs the models were built from; the full
arrays (12 MB for the Born gather) are not kept.  Run from the repository root after `make -C oracle`; takes a few
minutes on 8 cores:
    python tests/golden/make_config_golden.py
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

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "configs.npz")
STEP_C1, STEP_BORN, STEP_IMG = 16, 48, 8


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def rel(a, b) -> float:
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def dot_vectors(nx: int, nz: int, nt: int):
    rng = np.random.default_rng(22)
    m = rng.standard_normal((nx, nz)).astype(np.float32)
    d = rng.standard_normal((nx, nt)).astype(np.float32)
    return m, d


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libseisref.so is missing: run make -C oracle REF=...")
    O.ref_set_threads(os.cpu_count() or 1)
    out = {}
    t = time.time()
    c1 = synth.single_modeling()
    s1 = c1.shots[0]
    wav1 = O.ricker(s1.dt, c1.fr, s1.ndel, s1.NT, impl="ref")
    rec1 = O.modeling(s1, wav1, c1.vel, impl="ref")
    out.update(c1_vel_sha=sha(c1.vel), c1_wav_sha=sha(wav1), c1_rec_sha=sha(rec1),
               c1_rec_norm=np.linalg.norm(rec1.astype(np.float64)),
               c1_rec_sub=rec1[::STEP_C1].copy())
    print(f"config 1 modeling {time.time() - t:.1f} s, max|rec| {np.abs(rec1).max():.4g}")
    t = time.time()
    rec1_64 = O.modeling(s1, wav1.astype(np.float64), c1.vel, prec="f64")
    out.update(c1_rec_f64_sub=rec1_64[::STEP_C1].copy())
    print(f"config 1 modeling FP64 {time.time() - t:.1f} s, reference vs FP64 "
          f"{rel(rec1[::STEP_C1], rec1_64[::STEP_C1]):.3e}")

    t = time.time()
    c2 = synth.born_rtm_pair()
    s2 = c2.shots[0]
    wav2 = O.ricker(s2.dt, c2.fr, s2.ndel, s2.NT, impl="ref")
    born2 = O.born(s2, wav2, c2.vel0, c2.dv, impl="ref")
    print(f"config 2 Born {time.time() - t:.1f} s, max|born| {np.abs(born2).max():.4g}")
    t = time.time()
    born2_64 = O.born(s2, wav2.astype(np.float64), c2.vel0, c2.dv, prec="f64")
    out.update(c2_born_f64_sub=born2_64[::STEP_BORN].copy())
    print(f"config 2 Born FP64 {time.time() - t:.1f} s, reference vs FP64 "
          f"{rel(born2[::STEP_BORN], born2_64[::STEP_BORN]):.3e}")
    t = time.time()
    img2 = O.rtm(s2, wav2, c2.vel0, born2, impl="ref")
    print(f"config 2 RTM {time.time() - t:.1f} s, max|img| {np.abs(img2).max():.4g}")
    out.update(c2_vel_sha=sha(c2.vel), c2_vel0_sha=sha(c2.vel0), c2_wav_sha=sha(wav2),
               c2_born_sha=sha(born2), c2_born_norm=np.linalg.norm(born2.astype(np.float64)),
               c2_born_sub=born2[::STEP_BORN].copy(),
               c2_img_sha=sha(img2), c2_img_norm=np.linalg.norm(img2.astype(np.float64)),
               c2_img_sub=img2[::STEP_IMG].copy())

    t = time.time()
    m, d = dot_vectors(s2.nx, s2.nz, s2.nt)
    w64 = wav2.astype(np.float64)
    Lm = O.born(s2, w64, c2.vel0, m, prec="f64")
    Ltd = O.born_adjoint(s2, w64, c2.vel0, d, prec="f64")
    a = float(np.sum(Lm * d.astype(np.float64)))
    b = float(np.sum(m.astype(np.float64) * Ltd))
    out.update(c2_dot_fp64=np.array([a, b, np.linalg.norm(Lm), np.linalg.norm(d)]))
    print(f"config 2 FP64 dot test {time.time() - t:.1f} s: <Lm,d> {a!r} <m,LTd> {b!r} "
          f"rel {abs(a - b) / max(abs(a), abs(b)):.3e}")
    np.savez_compressed(OUT, **{k: np.asarray(v) for k, v in out.items()})
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
