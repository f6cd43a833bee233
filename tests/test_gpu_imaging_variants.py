"""The reference's Hilbert imaging variants on the GPU, bit for bit against
the oracle restatement (pinned to the compiled reference by
tests/test_oracle.py): rtm_true (src/util/fd.cpp:924-1052) and adjointUpDown
(src/util/fd.cpp:340-590)."""
import numpy as np
import pytest

import oracle as O
from helpers import fd_args, golden_cases, golden_ids
from seis_b200 import fd

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("g", golden_cases(), ids=golden_ids())
def test_rtm_true_golden_bit_exact(ctx, g):
    got = fd.rtm_true(*fd_args(g.shot), g.wav, g.vel, g.rec, ctx=ctx)
    want = O.rtm_true(g.shot, g.wav, g.vel, g.rec)
    assert np.array_equal(got, want)
    assert np.abs(want).max() > 0


@pytest.mark.parametrize("g", golden_cases(), ids=golden_ids())
def test_rtm_updown_golden_bit_exact(ctx, g):
    wavh = O.hilbert(g.wav, 30)
    img, comp = fd.rtm_updown(*fd_args(g.shot), g.wav, wavh, g.vel, g.rec, ctx=ctx)
    want_img, want_comp = O.rtm_updown(g.shot, g.wav, wavh, g.vel, g.rec)
    for k in range(4):
        assert np.array_equal(comp[k], want_comp[k]), f"component {k}"
    assert np.array_equal(img, want_img)
    assert np.abs(want_comp).max(axis=(1, 2)).min() > 0
