"""Shot batches on the GPU: uneven shots advancing in the same launches must
give each shot exactly its single-shot (reference) result, and plans replayed
from their CUDA graph must repeat their first run exactly."""
import numpy as np
import pytest

import oracle as O
from seis_b200 import Shot
from seis_b200._lib import (IN_DV, IN_GATHER, IN_VEL, IN_WAVELET, OP_BORN, OP_MODELING, OP_RTM,
                            OUT_GATHER, OUT_IMAGE, Plan, batch)

pytestmark = pytest.mark.gpu


def uneven_shots(seed, n, nt=120, ndel=20):
    rng = np.random.default_rng(seed)
    shots, vels, dvs = [], [], []
    for _ in range(n):
        nx, nz = int(rng.integers(30, 170)), int(rng.integers(12, 100))
        pml = int(rng.integers(4, 30))
        shots.append(Shot(nx=nx, nz=nz, pml=pml, nt=nt, ndel=ndel, sx=int(rng.integers(0, nx)),
                          sz=int(rng.integers(0, nz)), dt=1e-3, dx=float(rng.uniform(8, 14)),
                          dz=float(rng.uniform(8, 14)), gz=rng.integers(0, nz, nx)))
        vels.append((1500 + 2500 * rng.random((nx, nz))).astype(np.float32))
        dvs.append((rng.standard_normal((nx, nz)) * 40).astype(np.float32))
    wav = O.ricker(1e-3, 25.0, ndel, nt + ndel)
    return shots, vels, dvs, wav


def test_modeling_batch_matches_single_shots(ctx):
    shots, vels, _, wav = uneven_shots(11, 5)
    recs = batch(ctx, OP_MODELING, shots, [wav] * 5, vels)
    for s, v, r in zip(shots, vels, recs):
        assert np.array_equal(r, O.modeling(s, wav, v))


def test_born_batch_matches_single_shots(ctx):
    shots, vels, dvs, wav = uneven_shots(12, 4)
    recs = batch(ctx, OP_BORN, shots, [wav] * 4, vels, dvs)
    for s, v, d, r in zip(shots, vels, dvs, recs):
        assert np.array_equal(r, O.born(s, wav, v, d))


def test_rtm_batch_matches_single_shots(ctx):
    shots, vels, _, wav = uneven_shots(13, 3)
    recs = [O.modeling(s, wav, v) for s, v in zip(shots, vels)]
    imgs = batch(ctx, OP_RTM, shots, [wav] * 3, vels, recs)
    for s, v, r, img in zip(shots, vels, recs, imgs):
        assert np.array_equal(img, O.rtm(s, wav, v, r))


@pytest.mark.parametrize("op", [OP_MODELING, OP_BORN, OP_RTM])
def test_plan_graph_replay_is_repeatable(ctx, op):
    shots, vels, dvs, wav = uneven_shots(14, 3, nt=80, ndel=10)
    p = Plan(ctx, op, shots)
    for i, s in enumerate(shots):
        p.set(i, IN_VEL, vels[i])
        p.set(i, IN_WAVELET, wav)
        if op == OP_BORN:
            p.set(i, IN_DV, dvs[i])
        if op == OP_RTM:
            p.set(i, IN_GATHER, O.modeling(s, wav, vels[i]))
    what = OUT_IMAGE if op == OP_RTM else OUT_GATHER
    p.run()
    first = [p.get(i, what) for i in range(len(shots))]
    p.run()
    p.run()
    again = [p.get(i, what) for i in range(len(shots))]
    for a, b in zip(first, again):
        assert np.array_equal(a, b)
    assert p.launches_per_run > 0
    if op == OP_MODELING:
        for s, v, r in zip(shots, vels, first):
            assert np.array_equal(r, O.modeling(s, wav, v))
    p.close()


@pytest.mark.parametrize("op", [OP_MODELING, OP_BORN, OP_RTM])
def test_fast_flavour_within_fp32_gate(ctx, op):
    """Contracted arithmetic (exact=0): gathers within 1e-5 relative L2 of the
    reference (the FP32 gather gate); RTM images within 1e-5 too."""
    from helpers import rel_l2
    shots, vels, dvs, wav = uneven_shots(21, 3, nt=150, ndel=20)
    p = Plan(ctx, op, shots)
    p.set_exact(False)
    refs = []
    for i, s in enumerate(shots):
        p.set(i, IN_VEL, vels[i])
        p.set(i, IN_WAVELET, wav)
        if op == OP_MODELING:
            refs.append(O.modeling(s, wav, vels[i]))
        elif op == OP_BORN:
            p.set(i, IN_DV, dvs[i])
            refs.append(O.born(s, wav, vels[i], dvs[i]))
        else:
            rec = O.modeling(s, wav, vels[i])
            p.set(i, IN_GATHER, rec)
            refs.append(O.rtm(s, wav, vels[i], rec))
    p.run()
    what = OUT_IMAGE if op == OP_RTM else OUT_GATHER
    for i in range(len(shots)):
        assert rel_l2(p.get(i, what), refs[i]) < 1e-5
    p.close()
