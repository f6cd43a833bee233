"""The C-ABI library: it loads, exports every function include/*.h declares,
and its host-only entry points behave (no device needed)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import seis_b200
from seis_b200 import Shot
from seis_b200._lib import LIB_PATH, ricker, validate_shot

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(seis_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    names = declared_functions()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version():
    assert seis_b200.lib().seis_fd_abi_version() == 2


def test_ricker_matches_reference_wavelet():
    import oracle as O
    w = ricker(1e-3, 15.0, 100, 2100)
    assert np.array_equal(w, O.ricker(1e-3, 15.0, 100, 2100))


def base_shot(**kw):
    d = dict(nx=20, nz=10, pml=5, nt=10, ndel=2, sx=3, sz=1, dt=1e-3, dx=10.0, dz=10.0)
    d.update(kw)
    return Shot(**d)


def test_validate_accepts_good_shot():
    assert validate_shot(base_shot()) == ""


@pytest.mark.parametrize("kw,frag", [
    (dict(nx=0), "nx=0"),
    (dict(nt=0), "nt=0"),
    (dict(dt=0.0), "positive"),
    (dict(sx=-6), "source"),
    (dict(pml=0, sz=0), "source"),
    (dict(nx=2, nz=1, pml=1, sx=0, sz=0), "smaller than 5x5"),
])
def test_validate_rejects(kw, frag):
    assert frag in validate_shot(base_shot(**kw))


def test_validate_rejects_receiver_on_frame():
    s = base_shot()
    s.gz[3] = -5
    assert "gz[3]" in validate_shot(s)


def test_noalloc_dot_rejects_null_pointers_without_a_device():
    """seis_fd_vec_dot_noalloc checks its pointers before any CUDA call: null
    operands give SEIS_ERR_ARG with a message, and a null message buffer is
    accepted."""
    f = seis_b200.lib().seis_fd_vec_dot_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    f.restype = ctypes.c_int
    err = ctypes.create_string_buffer(128)
    fake = ctypes.c_void_p(0x1000)  # never dereferenced: the call fails first
    assert f(None, fake, 8, fake, None, err, len(err)) == -1
    assert b"null pointer" in err.value
    assert f(fake, fake, 8, None, None, err, len(err)) == -1
    assert b"null pointer" in err.value
    assert f(fake, None, 8, fake, None, None, 0) == -1
