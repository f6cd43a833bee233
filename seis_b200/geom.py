"""Per-shot acquisition geometry of the shot driver (include/seis_geom.h).

The reference keeps these as members of its MPI driver class ``Inversion``
(src/lsrtm/inversion.cpp:552-752); the library's versions are plain host
functions over flat arrays with the reference's float/double arithmetic.
Models are [nx][nz], gathers [ntrace][nt] (numpy, C order)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import SeisError, lib

_F = ctypes.c_float
_I = ctypes.c_int
_P = ctypes.c_void_p


def _setup():
    L = lib()
    if getattr(L, "_geom_ready", False):
        return L
    L.seis_geom_aperture.argtypes = [_F, _P, _I, _F, _I, _I, ctypes.POINTER(_F), ctypes.POINTER(_I)]
    L.seis_geom_extract.argtypes = [_P, _I, _I, _F, _F, _F, _I, _P]
    L.seis_geom_extract_columns.argtypes = [_I, _F, _F, _F, _I, _P]
    L.seis_geom_receiver_rows.argtypes = [_P, _P, _I, _F, _I, _F, _F, _I, _P]
    L.seis_geom_source_index.argtypes = [_F, _F, _F, _F, _F, ctypes.POINTER(_I), ctypes.POINTER(_I)]
    L.seis_geom_reorder.argtypes = [_P, _I, _I, _P, _P, _F, _I, _F, _I]
    L.seis_geom_swap_model.argtypes = [_P, _P, _F, _F, _I, _I, _I, _I, _F, _I]
    L.seis_geom_remove_direct.argtypes = [_P, _I, _I, _P, _P, _F, _F, _P, _I, _I, _F, _F, _F, _F,
                                          _F, _I]
    L._geom_ready = True
    return L


def _ok(rc, what):
    if rc != 0:
        raise SeisError(f"{what}: status {rc}")


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _p(a):
    return a.ctypes.data_as(_P)


def aperture(sx, gx, dx, lpad, rpad):
    """(fx_sub, nx_sub) of one shot (Inversion::getVel, inversion.cpp:552-568)."""
    L = _setup()
    g = _f32(gx)
    fx, nx = _F(), _I()
    _ok(L.seis_geom_aperture(sx, _p(g), len(g), dx, lpad, rpad, ctypes.byref(fx), ctypes.byref(nx)),
        "aperture")
    return fx.value, nx.value


def extract(model, fx, dx, fx_sub, nx_sub):
    """Sub-grid [nx_sub][nz] of model [nx][nz] (Inversion::getVel, :572-598)."""
    L = _setup()
    m = _f32(model)
    out = np.zeros((nx_sub, m.shape[1]), np.float32)
    _ok(L.seis_geom_extract(_p(m), m.shape[1], m.shape[0], fx, dx, fx_sub, nx_sub, _p(out)),
        "extract")
    return out


def extract_columns(nx, fx, dx, fx_sub, nx_sub):
    """Model column each sub-grid column copies (non-decreasing)."""
    L = _setup()
    out = np.zeros(nx_sub, np.int32)
    _ok(L.seis_geom_extract_columns(nx, fx, dx, fx_sub, nx_sub, _p(out)), "extract_columns")
    return out


def receiver_rows(gx, gz, fx_sub, nx_sub, dx, dz, nz):
    """Receiver depth index per sub-grid column (Inversion::getIgz, :600-625)."""
    L = _setup()
    x, z = _f32(gx), _f32(gz)
    out = np.zeros(nx_sub, np.int32)
    _ok(L.seis_geom_receiver_rows(_p(x), _p(z), len(x), fx_sub, nx_sub, dx, dz, nz, _p(out)),
        "receiver_rows")
    return out


def source_index(sx, sz, fx_sub, dx, dz):
    """Source sample indices in the sub-grid (inversion.cpp:428-429)."""
    L = _setup()
    a, b = _I(), _I()
    _ok(L.seis_geom_source_index(sx, sz, fx_sub, dx, dz, ctypes.byref(a), ctypes.byref(b)),
        "source_index")
    return a.value, b.value


def reorder_to_columns(csg, gx, fx, nx, dx):
    """rec [nx][nt] from traces csg [ng][nt] (Inversion::swapReord, adj=false)."""
    L = _setup()
    c = _f32(csg)
    rec = np.zeros((nx, c.shape[1]), np.float32)
    g = _f32(gx)
    _ok(L.seis_geom_reorder(_p(c), c.shape[0], c.shape[1], _p(g), _p(rec), fx, nx, dx, 0),
        "reorder")
    return rec


def reorder_to_gather(rec, gx, fx, dx):
    """Traces [ng][nt] from rec [nx][nt] (Inversion::swapReord, adj=true)."""
    L = _setup()
    r = _f32(rec)
    g = _f32(gx)
    csg = np.zeros((len(g), r.shape[1]), np.float32)
    _ok(L.seis_geom_reorder(_p(csg), len(g), r.shape[1], _p(g), _p(r), fx, r.shape[0], dx, 1),
        "reorder")
    return csg


def swap_model(m, d, mfx, dfx, dx, add=False):
    """Sub-grid image m into global d in place (Inversion::swapModel, :644-665)."""
    L = _setup()
    mm = _f32(m)
    assert d.dtype == np.float32 and d.flags.c_contiguous
    _ok(L.seis_geom_swap_model(_p(mm), _p(d), mfx, dfx, mm.shape[1], mm.shape[0], d.shape[1],
                               d.shape[0], dx, 1 if add else 0), "swap_model")
    return d


def remove_direct(csg, gx, gz, sx, sz, v, dx, dz, dt, fr, velfx, delay):
    """Direct-arrival mute of csg [ng][nt] in place (Inversion::removeDirect, :699-752)."""
    L = _setup()
    assert csg.dtype == np.float32 and csg.flags.c_contiguous
    x, z, vv = _f32(gx), _f32(gz), _f32(v)
    _ok(L.seis_geom_remove_direct(_p(csg), csg.shape[0], csg.shape[1], _p(x), _p(z), sx, sz, _p(vv),
                                  vv.shape[1], vv.shape[0], dx, dz, dt, fr, velfx, delay),
        "remove_direct")
    return csg
