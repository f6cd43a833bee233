"""seis_fd_vec_dot_noalloc: the CG dot product for callers that cannot
allocate device memory (an application that owns the whole device budget, a
plugin that must not bypass its host's memory pool, a loop that cannot afford
the synchronisation of cudaMalloc/cudaFree).  Its scratch is a fixed array
inside the library, so its result is checked against seis_fd_vec_dot on two
calls in a row, the second seeing whatever the first left in the scratch.

Collected last on purpose: the file name sorts after every other test file."""
import ctypes

import numpy as np
import pytest

from seis_b200._lib import lib

pytestmark = pytest.mark.gpu

MAX_N = 16384 * 4096  # SEIS_DOT_NOALLOC_MAX_N
SEIS_ERR_ARG = -1


def _noalloc():
    L = lib()
    f = L.seis_fd_vec_dot_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    f.restype = ctypes.c_int
    return f


def _ref_dot(ctx, a, b, n):
    out = ctypes.c_double()
    ctx.check(ctx.L.seis_fd_vec_dot(ctx.h, ctypes.c_void_p(a.data_ptr()),
                                    ctypes.c_void_p(b.data_ptr()), n, ctypes.byref(out)))
    return out.value


def _call(f, a, b, n, out, torch):
    err = ctypes.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = f(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), n,
           ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream), err, len(err))
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("n", [1, 4097, 3_000_001, MAX_N])
def test_noalloc_dot_matches_vec_dot_twice(ctx, n):
    import torch
    f = _noalloc()
    g = torch.Generator(device="cuda").manual_seed(n)
    a = torch.randn(n, device="cuda", generator=g)
    b = torch.randn(n, device="cuda", generator=g)
    c = torch.rand(n, device="cuda", generator=g)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for x, y in ((a, b), (b, c)):  # two calls in a row on the shared scratch
        got = _call(f, x, y, n, out, torch)
        want = _ref_dot(ctx, x, y, n)
        scale = float(torch.sum(torch.abs(x * y).double()).item())
        print(f"n={n}: noalloc {got!r} vec_dot {want!r}")
        assert abs(got - want) <= 1e-12 * scale, (got, want)


def test_noalloc_dot_rejects_oversize_and_empty(ctx):
    import torch
    f = _noalloc()
    a = torch.ones(8, device="cuda")
    out = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    err = ctypes.create_string_buffer(256)
    rc = f(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(a.data_ptr()), MAX_N + 1,
           ctypes.c_void_p(out.data_ptr()), None, err, len(err))
    assert rc == SEIS_ERR_ARG
    assert b"exceeds the maximum" in err.value
    assert _call(f, a, a, 0, out, torch) == 0.0
    assert _call(f, a, a, 8, out, torch) == 8.0
    assert np.isclose(_ref_dot(ctx, a, a, 8), 8.0)
