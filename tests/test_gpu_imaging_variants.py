"""The reference's Hilbert imaging variants on the GPU, bit for bit against
the oracle restatement (pinned to the compiled reference by
tests/test_oracle.py): rtm_true (src/util/fd.cpp:924-1052)."""
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
