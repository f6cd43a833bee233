"""ctypes binding of ``libseisfd.so`` (the C ABI of include/seis_fd.h).

The library is built in-tree by ``seis_b200.build``.  There is no CPU fallback:
if the library is missing or no CUDA device is present, the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libseisfd.so")

SEIS_OK = 0
ERRORS = {-1: "SEIS_ERR_ARG", -2: "SEIS_ERR_CUDA", -3: "SEIS_ERR_NOMEM", -4: "SEIS_ERR_STATE",
          -5: "SEIS_ERR_NOTSUP", -6: "SEIS_ERR_CANCELLED"}


class SeisError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class ShotDescC(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("nz", ctypes.c_int), ("pml", ctypes.c_int),
                ("nt", ctypes.c_int), ("ndel", ctypes.c_int), ("sx", ctypes.c_int),
                ("sz", ctypes.c_int), ("dt", ctypes.c_float), ("dx", ctypes.c_float),
                ("dz", ctypes.c_float), ("gz", ctypes.POINTER(ctypes.c_int))]


@dataclass
class Shot:
    """One shot: the scalar arguments of ``modeling``/``forward``/``adjoint``
    (src/util/fd.h:3-5) plus the receiver depths ``gz[nx]``."""
    nx: int
    nz: int
    pml: int
    nt: int
    ndel: int
    sx: int
    sz: int
    dt: float
    dx: float
    dz: float
    gz: np.ndarray = field(default=None)

    def __post_init__(self):
        if self.gz is None:
            self.gz = np.zeros(self.nx, np.int32)
        self.gz = np.ascontiguousarray(self.gz, np.int32)

    @property
    def NT(self) -> int:
        return self.nt + self.ndel

    def to_c(self) -> ShotDescC:
        d = ShotDescC(self.nx, self.nz, self.pml, self.nt, self.ndel, self.sx, self.sz,
                      self.dt, self.dx, self.dz,
                      self.gz.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        d._keep = self.gz  # keep the receiver array alive with the struct
        return d


_lib = None


def lib():
    """Load the library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m seis_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P, I = ctypes.c_void_p, ctypes.c_int
        SD = ctypes.POINTER(ShotDescC)
        L.seis_fd_abi_version.restype = I
        L.seis_fd_create.argtypes = [ctypes.POINTER(P), I]
        L.seis_fd_destroy.argtypes = [P]
        L.seis_fd_last_error.argtypes = [P]
        L.seis_fd_last_error.restype = ctypes.c_char_p
        L.seis_fd_launch_count.argtypes = [P]
        L.seis_fd_launch_count.restype = ctypes.c_int64
        L.seis_fd_ricker.argtypes = [ctypes.c_float, ctypes.c_float, I, I, P]
        L.seis_fd_validate_shot.argtypes = [SD, ctypes.c_char_p, ctypes.c_size_t]
        L.seis_fd_modeling.argtypes = [P, SD, P, P, P]
        L.seis_fd_born.argtypes = [P, SD, P, P, P, P]
        L.seis_fd_rtm.argtypes = [P, SD, P, P, P, P]
        _lib = L
    return _lib


def ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class Context:
    """One device context (one CUDA stream); mirrors seis_fd_create/destroy."""

    def __init__(self, device: int = 0):
        self.L = lib()
        h = ctypes.c_void_p()
        rc = self.L.seis_fd_create(ctypes.byref(h), device)
        if rc != SEIS_OK:
            raise SeisError(rc, f"seis_fd_create(device={device}) failed")
        self.h = h

    def check(self, rc: int):
        if rc != SEIS_OK:
            msg = self.L.seis_fd_last_error(self.h)
            raise SeisError(rc, msg.decode() if msg else "")

    @property
    def launches(self) -> int:
        return int(self.L.seis_fd_launch_count(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.L.seis_fd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def ricker(dt: float, fr: float, delay: int, n: int) -> np.ndarray:
    """Reference Ricker wavelet (src/util/wavelet.cpp:7-18), computed by the
    library's host code in the reference's single-precision arithmetic."""
    out = np.zeros(n, np.float32)
    rc = lib().seis_fd_ricker(dt, fr, delay, n, ptr(out))
    if rc != SEIS_OK:
        raise SeisError(rc, "seis_fd_ricker")
    return out


def validate_shot(shot: "Shot") -> str:
    """Host-only argument check of one shot; returns '' if valid, else the reason."""
    buf = ctypes.create_string_buffer(512)
    rc = lib().seis_fd_validate_shot(shot.to_c(), buf, 512)
    return "" if rc == SEIS_OK else (buf.value.decode() or f"error {rc}")
