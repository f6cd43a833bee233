"""B200-native 2-D acoustic finite-difference engine (forward, Born, RTM, LSRTM).

The compute path is the C-ABI library ``lib/libseisfd.so`` (CUDA, sm_100a),
declared in ``include/seis_fd.h``.  This package is its Python host mirror.
"""
from ._lib import Context, SeisError, Shot, lib  # noqa: F401
from . import fd  # noqa: F401

__all__ = ["Context", "SeisError", "Shot", "lib", "fd"]
