"""The C restatement (oracle/) at the sizes of the single-shot benchmark
configurations, against the reference's own outputs in
tests/golden/configs.npz (made by tests/golden/make_config_golden.py), and the
FP64 Born / exact-adjoint pair on the 737 x 240 grid."""
import hashlib
import os

import numpy as np

import oracle as O
from helpers import GOLDEN
from seis_b200 import synth


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def test_restatement_reproduces_config1_gather():
    gold = np.load(os.path.join(GOLDEN, "configs.npz"))
    c = synth.single_modeling()
    s = c.shots[0]
    assert sha(c.vel) == str(gold["c1_vel_sha"])
    wav = O.ricker(s.dt, c.fr, s.ndel, s.NT)
    assert sha(wav) == str(gold["c1_wav_sha"])
    rec = O.modeling(s, wav, c.vel)
    assert sha(rec) == str(gold["c1_rec_sha"])
    # the FP64 gather the GPU tests state the FP32 errors against
    rec64 = O.modeling(s, wav.astype(np.float64), c.vel, prec="f64")
    assert np.array_equal(rec64[::16], gold["c1_rec_f64_sub"])


def test_fp64_pair_is_a_transpose_on_the_737x240_grid():
    """The FP64 Born operator and its exact transpose on the full 737 x 240
    shot (nt cut to 400 to keep the CPU suite short; the fixture holds the
    full nt 4000 pair), seeded N(0, 1) vectors."""
    c = synth.born_rtm_pair(nt=400)
    s = c.shots[0]
    wav = O.ricker(s.dt, c.fr, s.ndel, s.NT).astype(np.float64)
    rng = np.random.default_rng(22)
    m = rng.standard_normal((s.nx, s.nz)).astype(np.float32)
    d = rng.standard_normal((s.nx, s.nt)).astype(np.float32)
    Lm = O.born(s, wav, c.vel0, m, prec="f64")
    Ltd = O.born_adjoint(s, wav, c.vel0, d, prec="f64")
    a = float(np.sum(Lm * d.astype(np.float64)))
    b = float(np.sum(m.astype(np.float64) * Ltd))
    assert abs(a - b) / (np.linalg.norm(Lm) * np.linalg.norm(d)) <= 1e-14
    assert abs(a - b) / max(abs(a), abs(b)) <= 1e-11
