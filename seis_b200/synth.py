"""Seeded synthetic models and acquisition geometries of the five workloads.

No public dataset is involved: every model is generated from numpy
``default_rng`` seeds, float32, in the reference layout ``[nx][nz]``
(z fastest).  Wavelets follow the reference ``rickerWavelet(dt, fr, delay, NT)``
(src/util/wavelet.cpp:7-18) with ``delay = ndel = ceil(1.5 / (fr dt))``.

Workloads (pml = 40 everywhere):

* ``single_modeling``  201x201 at 10 m, linear-gradient over a flat reflector,
  one shot, nt 2000, dt 1 ms, 15 Hz.
* ``born_rtm_pair``    737x240 at 12.5 m, 20 random layers, smooth background
  (Gaussian sigma 10 cells), reflectivity = true - smooth, nt 4000, 20 Hz.
* ``batched_rtm``      the layered model + 10 Gaussian anomalies, 64 shots of
  uneven aperture (300-737 columns).
* ``lsrtm``            1200x400 at 10 m, layers + 3 dipping faults, 32 shots,
  nt 5000, dt 0.8 ms.
* ``large_sweep``      4000x1000 at 5 m, layers + anomalies 1500-5500 m/s, 256
  shots of aperture 1000-4000, nt 8000, dt 0.5 ms, 25 Hz.

The module imports numpy and scipy only (no part of this package), so that a
CPU-only measurement of the reference can build the same inputs without
loading the CUDA library; its shot records carry the fields of the C ABI's
``seis_shot_desc`` and are accepted wherever a ``seis_b200.Shot`` is.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List

import numpy as np

PML = 40


@dataclass
class ShotGeom:
    """One shot's scalars (src/util/fd.h:3-5) and receiver depths ``gz[nx]``."""
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


def ndel_for(fr: float, dt: float) -> int:
    return int(math.ceil(1.5 / (fr * dt) - 1e-9))


def ricker(dt: float, fr: float, delay: int, n: int) -> np.ndarray:
    """Reference Ricker wavelet (src/util/wavelet.cpp:7-18), via the library."""
    from seis_b200._lib import ricker as _ricker
    return _ricker(dt, fr, delay, n)


@dataclass
class Survey:
    """A multi-shot experiment on one global model (the reference Inversion's
    view: global grid, one aperture sub-grid per shot)."""
    name: str
    nx: int
    nz: int
    dx: float
    dz: float
    dt: float
    nt: int
    fr: float
    vel: np.ndarray          # true velocity [nx][nz]
    vel0: np.ndarray         # smooth background [nx][nz]
    shots: List[ShotGeom]    # per-shot aperture descriptors
    x0: List[int]            # first global column of each aperture

    @property
    def ndel(self) -> int:
        return ndel_for(self.fr, self.dt)

    @property
    def dv(self) -> np.ndarray:
        return (self.vel - self.vel0).astype(np.float32)

    def wavelet(self, make=None) -> np.ndarray:
        """The survey's wavelet; ``make(dt, fr, delay, n)`` defaults to the
        library's ``seis_fd_ricker``."""
        return (make or ricker)(self.dt, self.fr, self.ndel, self.nt + self.ndel)

    def sub(self, a: np.ndarray, s: int) -> np.ndarray:
        """Aperture sub-model of shot s (columns x0 .. x0+nx)."""
        return np.ascontiguousarray(a[self.x0[s]:self.x0[s] + self.shots[s].nx], np.float32)

    def cell_updates_of(self, i: int) -> int:
        s = self.shots[i]
        return (s.nx + 2 * s.pml) * (s.nz + 2 * s.pml) * s.NT

    def subset(self, idx) -> "Survey":
        """The same survey restricted to shots idx."""
        idx = list(idx)
        return Survey(self.name, self.nx, self.nz, self.dx, self.dz, self.dt, self.nt, self.fr,
                      self.vel, self.vel0, [self.shots[i] for i in idx], [self.x0[i] for i in idx])

    def cell_updates(self, fields: int = 1) -> int:
        return sum((s.nx + 2 * s.pml) * (s.nz + 2 * s.pml) * s.NT for s in self.shots) * fields


def _layers(nx, nz, nlayers, rng, vmin, vmax):
    vals = np.sort(rng.uniform(vmin, vmax, nlayers))
    thick = nz // nlayers
    v = np.empty((nx, nz), np.float64)
    for k in range(nlayers):
        z1 = nz if k == nlayers - 1 else (k + 1) * thick
        v[:, k * thick:z1] = vals[k]
    return v


def _smooth(v, sigma=10.0):
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(v, sigma=sigma, mode="nearest")


def _anomalies(v, n, rng, amp=300.0, rmin=5, rmax=20):
    nx, nz = v.shape
    X, Z = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    for _ in range(n):
        cx, cz = rng.uniform(0, nx), rng.uniform(0, nz)
        r = rng.uniform(rmin, rmax)
        a = rng.choice([-1.0, 1.0]) * amp
        v = v + a * np.exp(-((X - cx) ** 2 + (Z - cz) ** 2) / (2 * r * r))
    return v


def _shot(nx_sub, nz, sx, sz, gz, dt, dx, dz, nt, fr, pml=PML) -> ShotGeom:
    return ShotGeom(nx=nx_sub, nz=nz, pml=pml, nt=nt, ndel=ndel_for(fr, dt), sx=sx, sz=sz,
                dt=dt, dx=dx, dz=dz, gz=np.full(nx_sub, gz, np.int32))


def single_modeling(nt: int = 2000) -> Survey:
    nx = nz = 201
    dx = dz = 10.0
    z = np.arange(nz) * dz
    col = np.where(z < 1000.0, 2000.0 + 0.5 * z, 3000.0)
    v = np.tile(col, (nx, 1)).astype(np.float32)
    shot = _shot(nx, nz, 100, 2, 2, 1e-3, dx, dz, nt, 15.0)
    return Survey("single_modeling", nx, nz, dx, dz, 1e-3, nt, 15.0, v, v.copy(), [shot], [0])


def layered_737(seed: int = 2):
    nx, nz = 737, 240
    v = _layers(nx, nz, 20, np.random.default_rng(seed), 1500.0, 4500.0)
    return v, _smooth(v)


def born_rtm_pair(nt: int = 4000) -> Survey:
    v, v0 = layered_737()
    nx, nz = v.shape
    shot = _shot(nx, nz, 368, 1, 1, 1e-3, 12.5, 12.5, nt, 20.0)
    return Survey("born_rtm_pair", nx, nz, 12.5, 12.5, 1e-3, nt, 20.0, v.astype(np.float32),
                  v0.astype(np.float32), [shot], [0])


def batched_rtm(nshots: int = 64, nt: int = 4000) -> Survey:
    v, _ = layered_737()
    rng = np.random.default_rng(3)
    v = _anomalies(v, 10, rng)
    v0 = _smooth(v)
    nx, nz = v.shape
    widths = rng.integers(300, 738, nshots)
    shots, x0s = [], []
    for w in widths:
        w = int(w)
        x0 = int(rng.integers(0, nx - w + 1))
        shots.append(_shot(w, nz, w // 2, 1, 1, 1e-3, 12.5, 12.5, nt, 20.0))
        x0s.append(x0)
    return Survey("batched_rtm", nx, nz, 12.5, 12.5, 1e-3, nt, 20.0, v.astype(np.float32),
                  v0.astype(np.float32), shots, x0s)


def _faults(v, rng, dz, nfault=3):
    nx, nz = v.shape
    out = v.copy()
    X = np.arange(nx)
    for _ in range(nfault):
        xc = rng.uniform(0.2 * nx, 0.8 * nx)
        dip = rng.uniform(0.5, 2.0) * rng.choice([-1.0, 1.0])
        throw = int(round(rng.uniform(20.0, 60.0) / dz))
        for ix in X:
            # hanging wall: columns right of the dipping plane move down by `throw`
            zcut = int(np.clip((ix - xc) * dip + nz / 2, 0, nz))
            if ix > xc:
                col = out[ix].copy()
                out[ix, zcut:] = np.concatenate([np.repeat(col[zcut:zcut + 1], throw),
                                                 col[zcut:]])[:nz - zcut]
    return out


def lsrtm(nshots: int = 32, nt: int = 5000) -> Survey:
    nx, nz, dx = 1200, 400, 10.0
    rng = np.random.default_rng(4)
    v = _layers(nx, nz, 20, rng, 1500.0, 4500.0)
    v = _faults(v, rng, dx)
    v0 = _smooth(v)
    shots, x0s = [], []
    for i in range(nshots):
        sx = int((i + 0.5) * nx / nshots)
        shots.append(_shot(nx, nz, sx, 1, 1, 8e-4, dx, dx, nt, 20.0))
        x0s.append(0)
    return Survey("lsrtm", nx, nz, dx, dx, 8e-4, nt, 20.0, v.astype(np.float32),
                  v0.astype(np.float32), shots, x0s)


def large_sweep(nshots: int = 256, nt: int = 8000, vmax: float = 5500.0) -> Survey:
    """At vmax = 5500 m/s the Courant number v dt / dx reaches 0.55.  Over
    this survey's 8120 steps with its 40-cell pad the reference's scheme (its
    absorbing boundary; the interior 8th-order update alone is stable up to
    0.5546) grows without bound from a Courant number of about 0.33 up; vmax =
    3000 (0.30) runs stable."""
    nx, nz, dx = 4000, 1000, 5.0
    rng = np.random.default_rng(5)
    v = _layers(nx, nz, 20, rng, 1500.0, 5000.0)
    v = _anomalies(v, 20, rng, amp=300.0, rmin=10, rmax=40)
    v = np.clip(v, 1500.0, vmax)
    v0 = _smooth(v)
    widths = rng.integers(1000, 4001, nshots)
    shots, x0s = [], []
    for w in widths:
        w = int(w)
        x0 = int(rng.integers(0, nx - w + 1))
        shots.append(_shot(w, nz, w // 2, 1, 1, 5e-4, dx, dx, nt, 25.0))
        x0s.append(x0)
    return Survey("large_sweep", nx, nz, dx, dx, 5e-4, nt, 25.0, v.astype(np.float32),
                  v0.astype(np.float32), shots, x0s)
