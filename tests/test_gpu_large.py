"""One shot of the largest survey (4000 x 1000 cells at 5 m, nt 8000 + 120,
velocities capped at 3000 m/s; shot 64 of 256, 1137 columns) against the FP64
image of tests/golden/large_fp64.npz (made by tests/golden/make_large_fp64.py
from the reference's own Born data and the restatement's double build): the
first CG gradient L^T d of the exact adjoint, with the benchmark's storage
(FP16 source-term snapshots every 4 steps, source-field checkpoints every 256
steps), with BF16 ones, and with FP32 snapshots at every step, all within
1e-3 relative L2 of the FP64 image (on the fixture's every-4th-cell
subsample)."""
import hashlib
import os

import numpy as np
import pytest

from helpers import GOLDEN, rel_l2
from seis_b200 import synth
from seis_b200._lib import (IN_DV, IN_GATHER, IN_VEL, IN_WAVELET, OP_BORN, OP_BORN_ADJOINT,
                            OUT_GATHER, OUT_IMAGE, SNAP_BF16, SNAP_F16, SNAP_F32, Plan)

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def shot(ctx):
    g = np.load(os.path.join(GOLDEN, "large_fp64.npz"))
    sv = synth.large_sweep(vmax=3000.0)
    k = int(g["shot"])
    s = sv.shots[k]
    vel0, dv, wav = sv.sub(sv.vel0, k), sv.sub(sv.dv, k), sv.wavelet()
    assert (sha(vel0), sha(dv), sha(wav)) == (str(g["vel0_sha"]), str(g["dv_sha"]),
                                              str(g["wav_sha"]))
    with Plan(ctx, OP_BORN, [s]) as p:  # exact build: the reference's Born data
        p.set(0, IN_VEL, vel0)
        p.set(0, IN_DV, dv)
        p.set(0, IN_WAVELET, wav)
        p.run()
        d = p.get(0, OUT_GATHER)
    assert sha(d) == str(g["data_sha"])
    return g, s, vel0, wav, d


@pytest.mark.parametrize("every,dtype,ck", [(4, SNAP_F16, 256), (4, SNAP_BF16, 256),
                                            (1, SNAP_F32, 256)],
                         ids=["f16_every4_ck256", "bf16_every4_ck256", "f32_every1_ck256"])
def test_large_shot_image_vs_fp64(ctx, shot, every, dtype, ck):
    g, s, vel0, wav, d = shot
    with Plan(ctx, OP_BORN_ADJOINT, [s]) as p:
        p.set_snapshots(every, dtype)
        p.set_checkpoints(ck)
        p.set(0, IN_VEL, vel0)
        p.set(0, IN_WAVELET, wav)
        p.set(0, IN_GATHER, d)
        p.run()
        img = p.get(0, OUT_IMAGE)
    st = int(g["step"])
    err = rel_l2(img[::st, ::st], g["img_sub"])
    print(f"every {every} dtype {dtype}: image rel L2 vs FP64 {err:.2e}")
    assert np.isfinite(img).all() and err <= 1e-3
