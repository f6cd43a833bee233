"""Python mirror of the reference propagator call surface (src/util/fd.h:3-5).

``modeling``, ``forward`` and ``adjoint`` take the reference's arguments in the
reference's order and return numpy arrays in the reference's layout
(gathers ``[nx][nt]``, images ``[nx][nz]``).  Each call runs on the GPU through
the C ABI; there is no CPU fallback.
"""
from __future__ import annotations

import numpy as np

from ._lib import Context, Shot, ptr

_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _shot(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz) -> Shot:
    return Shot(nx=nx, nz=nz, pml=pml, nt=nt, ndel=ndel, sx=sx, sz=sz, dt=dt, dx=dx, dz=dz, gz=gz)


def _f32(a, shape):
    a = np.ascontiguousarray(a, np.float32)
    if a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def modeling(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz, wav, vel, ctx: Context = None):
    """Shot gather ``rec[nx][nt]`` (reference ``modeling``, src/util/fd.cpp:15-80)."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz)
    wav = _f32(wav, (s.NT,))
    vel = _f32(vel, (nx, nz))
    rec = np.zeros((nx, nt), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_modeling(ctx.h, d, ptr(wav), ptr(vel), ptr(rec)))
    return rec


def forward_plane(dt, dx, dz, nt, ndel, nx, nz, pml, sz, gz, vel, sou, dv, ctx: Context = None):
    """Born gather ``rec[nx][nt]`` of the areal source ``sou[nx][nt+ndel]`` at row sz,
    receivers at row gz (reference ``forwordPlane``, src/util/fd.cpp:178-274)."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, nx // 2, sz, np.full(nx, gz, np.int32))
    sou = _f32(sou, (nx, s.NT))
    vel = _f32(vel, (nx, nz))
    dv = _f32(dv, (nx, nz))
    rec = np.zeros((nx, nt), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_born_plane(ctx.h, d, ptr(sou), ptr(vel), ptr(dv), ptr(rec)))
    return rec


def rtm_true(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz, wav, vel, rec, ctx: Context = None):
    """Image ``img[nx][nz]`` of the reference ``rtm_true`` (src/util/fd.cpp:924-1052):
    dipole receiver injection, FaQi imaging of the source field."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz)
    wav = _f32(wav, (s.NT,))
    vel = _f32(vel, (nx, nz))
    rec = _f32(rec, (nx, nt))
    img = np.zeros((nx, nz), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_rtm_true(ctx.h, d, ptr(wav), ptr(vel), ptr(rec), ptr(img)))
    return img


def rtm_updown(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz, wav, wavh, vel, rec,
               ctx: Context = None):
    """Image ``img[nx][nz]`` and components ``comp[4][nx][nz]`` of the reference
    ``adjointUpDown`` (src/util/fd.cpp:340-590).  ``wavh`` is the Hilbert transform
    of ``wav`` (the reference's caller filters the first nt samples with 100
    half-taps, src/lsrtm/lsrtm.cpp:97-99; see ``hilbert``); comp = (S R, H[S] H[R],
    St H[R], H[St] R) summed over the reverse pass (the model cells of the
    reference's padded imagX) and img = comp0 - comp1 + comp3 + comp2."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz)
    wav = _f32(wav, (s.NT,))
    wavh = _f32(wavh, (s.NT,))
    vel = _f32(vel, (nx, nz))
    rec = _f32(rec, (nx, nt))
    img = np.zeros((nx, nz), np.float32)
    comp = np.zeros((4, nx, nz), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_rtm_updown(ctx.h, d, ptr(wav), ptr(wavh), ptr(vel), ptr(rec),
                                       ptr(img), ptr(comp)))
    return img, comp


def adjoint_plane(dt, dx, dz, nt, ndel, nx, nz, pml, sz, gz, vel, sou, rec, ctx: Context = None):
    """Image ``img[nx][nz]`` of the areal source ``sou[nx][nt+ndel]`` and the gather
    ``rec[nx][nt]`` at row gz (reference ``adjointPlane``, src/util/fd.cpp:787-921)."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, nx // 2, sz, np.full(nx, gz, np.int32))
    sou = _f32(sou, (nx, s.NT))
    vel = _f32(vel, (nx, nz))
    rec = _f32(rec, (nx, nt))
    img = np.zeros((nx, nz), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_rtm_plane(ctx.h, d, ptr(sou), ptr(vel), ptr(rec), ptr(img)))
    return img


def illum(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, wav, vel, ctx: Context = None):
    """Source illumination ``ss[nx][nz]`` (reference ``illum``, src/util/fd.cpp:275-339)."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, np.zeros(nx, np.int32))
    wav = _f32(wav, (s.NT,))
    vel = _f32(vel, (nx, nz))
    ss = np.zeros((nx, nz), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_illum(ctx.h, d, ptr(wav), ptr(vel), ptr(ss)))
    return ss


def illum_plane(dt, dx, dz, nt, ndel, nx, nz, pml, sz, vel, sou, ctx: Context = None):
    """Illumination ``ss[nx][nz]`` of the areal source ``sou[nx][nt+ndel]`` at row sz
    (reference ``illumPlane``, src/util/fd.cpp:720-786)."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, nx // 2, sz, np.zeros(nx, np.int32))
    sou = _f32(sou, (nx, s.NT))
    vel = _f32(vel, (nx, nz))
    ss = np.zeros((nx, nz), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_illum_plane(ctx.h, d, ptr(sou), ptr(vel), ptr(ss)))
    return ss


def forward(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz, wav, vel, dv, ctx: Context = None):
    """Born gather ``rec[nx][nt]`` (reference ``forward``, src/util/fd.cpp:81-177)."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz)
    wav = _f32(wav, (s.NT,))
    vel = _f32(vel, (nx, nz))
    dv = _f32(dv, (nx, nz))
    rec = np.zeros((nx, nt), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_born(ctx.h, d, ptr(wav), ptr(vel), ptr(dv), ptr(rec)))
    return rec


def adjoint(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz, wav, vel, rec, ctx: Context = None):
    """RTM image ``img[nx][nz]`` (reference ``adjoint``, src/util/fd.cpp:592-719)."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz)
    wav = _f32(wav, (s.NT,))
    vel = _f32(vel, (nx, nz))
    rec = _f32(rec, (nx, nt))
    img = np.zeros((nx, nz), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_rtm(ctx.h, d, ptr(wav), ptr(vel), ptr(rec), ptr(img)))
    return img


def born_adjoint(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz, wav, vel, rec,
                 ctx: Context = None):
    """Exact adjoint of ``forward`` (no reference counterpart): ``img[nx][nz]``
    with <forward(m), rec> = <m, born_adjoint(rec)> to FP32 rounding."""
    ctx = ctx or default_context()
    s = _shot(dt, dx, dz, nt, ndel, nx, nz, pml, sx, sz, gz)
    wav = _f32(wav, (s.NT,))
    vel = _f32(vel, (nx, nz))
    rec = _f32(rec, (nx, nt))
    img = np.zeros((nx, nz), np.float32)
    d = s.to_c()
    ctx.check(ctx.L.seis_fd_born_adjoint(ctx.h, d, ptr(wav), ptr(vel), ptr(rec), ptr(img)))
    return img
