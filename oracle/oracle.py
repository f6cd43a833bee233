"""ctypes front-end of the CPU oracles -- TEST INFRASTRUCTURE ONLY.

Two libraries, both built by ``oracle/Makefile``:

* ``_build/libseisoracle.so`` -- the plain-C restatement of the reference FD path
  (``seis_oracle_body.h``) in float (``prec="f32"``) and double (``prec="f64"``).
* ``_ref/libseisref.so`` -- the reference's own ``src/util/fd.cpp`` and helpers,
  compiled in place (present only where the reference sources were available at
  build time; the built file travels with the repository snapshot).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
import this module.  The product library never calls it.

Array conventions follow the reference (``src/util/memory.h:29-44``): models and
images ``[nx][nz]`` (z fastest), gathers ``[nx][nt]`` (t fastest), all C-ordered
numpy arrays.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libseisoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libseisref.so")

_P = ctypes.c_void_p
_I = ctypes.c_int


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _dtype(prec: str):
    return {"f32": np.float32, "f64": np.float64}[prec]


class _Lib:
    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
        self.lib = ctypes.CDLL(path)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = _Lib(ORACLE_SO).lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = _Lib(REF_SO).lib
    return _ref


# --------------------------------------------------------------------------
# restatement (orc_*)
# --------------------------------------------------------------------------
def _real(prec):
    return ctypes.c_float if prec == "f32" else ctypes.c_double


def ricker(dt, fr, delay, n, prec="f32", impl="oracle"):
    if impl == "ref":
        out = np.zeros(n, np.float32)
        F = ctypes.c_float
        ref_lib().ref_ricker(F(dt), F(fr), _I(delay), _I(n), _ptr(out))
        return out
    R = _real(prec)
    out = np.zeros(n, _dtype(prec))
    getattr(oracle_lib(), f"orc_ricker_{prec}")(R(dt), R(fr), _I(delay), _I(n), _ptr(out))
    return out


def set_abs(nz, nx, pml, prec="f32", impl="oracle"):
    out = np.zeros((nx + 2 * pml, nz + 2 * pml), _dtype(prec) if impl == "oracle" else np.float32)
    if impl == "ref":
        ref_lib().ref_set_abs(_I(nz), _I(nx), _I(pml), _ptr(out))
    else:
        getattr(oracle_lib(), f"orc_set_abs_{prec}")(_I(nz), _I(nx), _I(pml), _ptr(out))
    return out


def set_vel(v, pml, prec="f32", impl="oracle"):
    nx, nz = v.shape
    dt = _dtype(prec) if impl == "oracle" else np.float32
    v = np.ascontiguousarray(v, dt)
    out = np.zeros((nx + 2 * pml, nz + 2 * pml), dt)
    if impl == "ref":
        ref_lib().ref_set_vel(_ptr(v), _I(nz), _I(nx), _I(pml), _ptr(out))
    else:
        getattr(oracle_lib(), f"orc_set_vel_{prec}")(_ptr(v), _I(nz), _I(nx), _I(pml), _ptr(out))
    return out


def hilbert(x, half=30, prec="f32", impl="oracle"):
    dt = _dtype(prec) if impl == "oracle" else np.float32
    x = np.ascontiguousarray(x, dt)
    out = np.zeros_like(x)
    if impl == "ref":
        ref_lib().ref_hilbert(_ptr(x), _ptr(out), _I(x.size), _I(half))
    else:
        getattr(oracle_lib(), f"orc_hilbert_{prec}")(_ptr(x), _ptr(out), _I(x.size), _I(half))
    return out


def _common_args(shot, prec):
    R = _real(prec) if prec else ctypes.c_float
    s = shot
    return [R(s.dt), R(s.dx), R(s.dz), _I(s.nt), _I(s.ndel), _I(s.nx), _I(s.nz), _I(s.pml),
            _I(s.sx), _I(s.sz)]


def _prep(shot, prec, impl, *arrays):
    dt = np.float32 if impl == "ref" else _dtype(prec)
    gz = np.ascontiguousarray(shot.gz, np.int32)
    out = [gz] + [np.ascontiguousarray(a, dt) for a in arrays]
    return dt, out


def modeling(shot, wav, vel, prec="f32", impl="oracle"):
    """Shot gather [nx][nt] of ``modeling`` (src/util/fd.cpp:15-80)."""
    dt, (gz, wav, vel) = _prep(shot, prec, impl, wav, vel)
    rec = np.zeros((shot.nx, shot.nt), dt)
    if impl == "ref":
        rc = ref_lib().ref_modeling(*_common_args(shot, None), _ptr(gz), _ptr(wav), _ptr(vel), _ptr(rec))
    else:
        rc = getattr(oracle_lib(), f"orc_modeling_{prec}")(*_common_args(shot, prec), _ptr(gz),
                                                           _ptr(wav), _ptr(vel), _ptr(rec))
    if rc != 0:
        raise RuntimeError(f"oracle modeling failed ({rc})")
    return rec


def born_plane(shot, sou, vel, dv, gz, prec="f32", impl="oracle"):
    """Scattered gather [nx][nt] of ``forwordPlane`` (src/util/fd.cpp:178-274):
    areal source sou [nx][nt+ndel] at row shot.sz, receivers at row gz."""
    dt, (_, sou, vel, dv) = _prep(shot, prec, impl, sou, vel, dv)
    rec = np.zeros((shot.nx, shot.nt), dt)
    R = _real(prec) if impl != "ref" else ctypes.c_float
    s = shot
    args = [R(s.dt), R(s.dx), R(s.dz), _I(s.nt), _I(s.ndel), _I(s.nx), _I(s.nz), _I(s.pml),
            _I(s.sz), _I(int(gz))]
    if impl == "ref":
        rc = ref_lib().ref_born_plane(*args, _ptr(sou), _ptr(vel), _ptr(dv), _ptr(rec))
    else:
        rc = getattr(oracle_lib(), f"orc_born_plane_{prec}")(*args, _ptr(sou), _ptr(vel), _ptr(dv),
                                                             _ptr(rec))
    if rc != 0:
        raise RuntimeError(f"oracle born_plane failed ({rc})")
    return rec


def rtm_true(shot, wav, vel, rec, prec="f32", impl="oracle"):
    """Image [nx][nz] of ``rtm_true`` (src/util/fd.cpp:924-1052)."""
    dt, (gz, wav, vel, rec) = _prep(shot, prec, impl, wav, vel, rec)
    img = np.zeros((shot.nx, shot.nz), dt)
    if impl == "ref":
        rc = ref_lib().ref_rtm_true(*_common_args(shot, None), _ptr(gz), _ptr(wav), _ptr(vel),
                                    _ptr(rec), _ptr(img))
    else:
        rc = getattr(oracle_lib(), f"orc_rtm_true_{prec}")(*_common_args(shot, prec), _ptr(gz),
                                                           _ptr(wav), _ptr(vel), _ptr(rec),
                                                           _ptr(img))
    if rc != 0:
        raise RuntimeError(f"oracle rtm_true failed ({rc})")
    return img


def rtm_updown(shot, wav, wavh, vel, rec, prec="f32", impl="oracle"):
    """(image [nx][nz], components [4][nx][nz]) of ``adjointUpDown``
    (src/util/fd.cpp:340-591); components in imagX order 00, zz, tz, zt."""
    dt, (gz, wav, wavh, vel, rec) = _prep(shot, prec, impl, wav, wavh, vel, rec)
    img = np.zeros((shot.nx, shot.nz), dt)
    comp = np.zeros((4, shot.nx, shot.nz), dt)
    if impl == "ref":
        rc = ref_lib().ref_rtm_updown(*_common_args(shot, None), _ptr(gz), _ptr(wav), _ptr(wavh),
                                      _ptr(vel), _ptr(rec), _ptr(img), _ptr(comp))
    else:
        rc = getattr(oracle_lib(), f"orc_rtm_updown_{prec}")(*_common_args(shot, prec), _ptr(gz),
                                                             _ptr(wav), _ptr(wavh), _ptr(vel),
                                                             _ptr(rec), _ptr(img), _ptr(comp))
    if rc != 0:
        raise RuntimeError(f"oracle rtm_updown failed ({rc})")
    return img, comp


def rtm_plane(shot, sou, vel, rec, gz, prec="f32", impl="oracle"):
    """Image [nx][nz] of ``adjointPlane`` (src/util/fd.cpp:787-921): areal source
    sou [nx][nt+ndel] at row shot.sz, receivers rec [nx][nt] at row gz."""
    dt, (_, sou, vel, rec) = _prep(shot, prec, impl, sou, vel, rec)
    img = np.zeros((shot.nx, shot.nz), dt)
    R = _real(prec) if impl != "ref" else ctypes.c_float
    s = shot
    args = [R(s.dt), R(s.dx), R(s.dz), _I(s.nt), _I(s.ndel), _I(s.nx), _I(s.nz), _I(s.pml),
            _I(s.sz), _I(int(gz))]
    if impl == "ref":
        rc = ref_lib().ref_rtm_plane(*args, _ptr(sou), _ptr(vel), _ptr(rec), _ptr(img))
    else:
        rc = getattr(oracle_lib(), f"orc_rtm_plane_{prec}")(*args, _ptr(sou), _ptr(vel),
                                                            _ptr(rec), _ptr(img))
    if rc != 0:
        raise RuntimeError(f"oracle rtm_plane failed ({rc})")
    return img


def illum(shot, wav, vel, prec="f32", impl="oracle"):
    """Source illumination [nx][nz] of ``illum`` (src/util/fd.cpp:275-339)."""
    dt, (gz, wav, vel) = _prep(shot, prec, impl, wav, vel)
    ss = np.zeros((shot.nx, shot.nz), dt)
    if impl == "ref":
        rc = ref_lib().ref_illum(*_common_args(shot, None), _ptr(wav), _ptr(vel), _ptr(ss))
    else:
        rc = getattr(oracle_lib(), f"orc_illum_{prec}")(*_common_args(shot, prec), _ptr(wav),
                                                        _ptr(vel), _ptr(ss))
    if rc != 0:
        raise RuntimeError(f"oracle illum failed ({rc})")
    return ss


def illum_plane(shot, sou, vel, prec="f32", impl="oracle"):
    """Illumination [nx][nz] of ``illumPlane`` (src/util/fd.cpp:720-786): areal
    source sou [nx][nt+ndel] at row shot.sz."""
    dt, (_, sou, vel) = _prep(shot, prec, impl, sou, vel)
    ss = np.zeros((shot.nx, shot.nz), dt)
    R = _real(prec) if impl != "ref" else ctypes.c_float
    s = shot
    args = [R(s.dt), R(s.dx), R(s.dz), _I(s.nt), _I(s.ndel), _I(s.nx), _I(s.nz), _I(s.pml),
            _I(s.sz)]
    if impl == "ref":
        rc = ref_lib().ref_illum_plane(*args, _ptr(sou), _ptr(vel), _ptr(ss))
    else:
        rc = getattr(oracle_lib(), f"orc_illum_plane_{prec}")(*args, _ptr(sou), _ptr(vel), _ptr(ss))
    if rc != 0:
        raise RuntimeError(f"oracle illum_plane failed ({rc})")
    return ss


def born(shot, wav, vel, dv, prec="f32", impl="oracle"):
    """Scattered gather [nx][nt] of ``forward`` (src/util/fd.cpp:81-177)."""
    dt, (gz, wav, vel, dv) = _prep(shot, prec, impl, wav, vel, dv)
    rec = np.zeros((shot.nx, shot.nt), dt)
    if impl == "ref":
        rc = ref_lib().ref_born(*_common_args(shot, None), _ptr(gz), _ptr(wav), _ptr(vel), _ptr(dv),
                                _ptr(rec))
    else:
        rc = getattr(oracle_lib(), f"orc_born_{prec}")(*_common_args(shot, prec), _ptr(gz), _ptr(wav),
                                                       _ptr(vel), _ptr(dv), _ptr(rec))
    if rc != 0:
        raise RuntimeError(f"oracle born failed ({rc})")
    return rec


def rtm(shot, wav, vel, rec, prec="f32", impl="oracle"):
    """Image [nx][nz] of the reference ``adjoint`` (src/util/fd.cpp:592-719)."""
    dt, (gz, wav, vel, rec) = _prep(shot, prec, impl, wav, vel, rec)
    img = np.zeros((shot.nx, shot.nz), dt)
    if impl == "ref":
        rc = ref_lib().ref_rtm(*_common_args(shot, None), _ptr(gz), _ptr(wav), _ptr(vel), _ptr(rec),
                               _ptr(img))
    else:
        rc = getattr(oracle_lib(), f"orc_rtm_{prec}")(*_common_args(shot, prec), _ptr(gz), _ptr(wav),
                                                      _ptr(vel), _ptr(rec), _ptr(img))
    if rc != 0:
        raise RuntimeError(f"oracle rtm failed ({rc})")
    return img


def born_adjoint(shot, wav, vel, rec, prec="f64", every=1):
    """Image [nx][nz] of the exact transpose of ``born`` (the library's own
    adjoint; the reference has no exact adjoint to compare with).  With
    ``every`` > 1 the imaging sum keeps every ``every``-th step of the source
    term plus the last one, with trapezoid weights."""
    dt, (gz, wav, vel, rec) = _prep(shot, prec, "oracle", wav, vel, rec)
    img = np.zeros((shot.nx, shot.nz), dt)
    rc = getattr(oracle_lib(), f"orc_born_adjoint_thin_{prec}")(
        *_common_args(shot, prec), _ptr(gz), _ptr(wav), _ptr(vel), _ptr(rec), _I(every), _ptr(img))
    if rc != 0:
        raise RuntimeError(f"oracle born_adjoint failed ({rc})")
    return img


def born_adjoint_ck(shot, wav, vel, rec, ck, prec="f64"):
    """born_adjoint with every = 1 in bounded memory: the source terms are
    recomputed per ck-step segment from checkpoints (the same image)."""
    dt, (gz, wav, vel, rec) = _prep(shot, prec, "oracle", wav, vel, rec)
    img = np.zeros((shot.nx, shot.nz), dt)
    rc = getattr(oracle_lib(), f"orc_born_adjoint_ck_{prec}")(
        *_common_args(shot, prec), _ptr(gz), _ptr(wav), _ptr(vel), _ptr(rec), _I(ck), _ptr(img))
    if rc != 0:
        raise RuntimeError(f"oracle born_adjoint_ck failed ({rc})")
    return img


def lsrtm_cgls(nx, nz, shots, x0, wav, v0, dobs, niter, prec="f64", cols=None):
    """CGLS on the global model (the solver the reference declares as
    Inversion::conope_MPI / cgsolver_MPI, src/lsrtm/inversion.h:81,87, without
    a definition), built from the oracle's Born operator and its exact
    transpose, in FP64.  Shot k covers model columns x0[k] .. x0[k]+nx_k-1, or
    the columns cols[k] (a sub-grid column map, repeated columns summed by the
    transpose).  Returns (model, |d|^2, [|r|^2 after each iteration])."""
    f = np.float64
    wav = np.asarray(wav, f)
    if cols is None:
        cols = [np.arange(x, x + s.nx) for s, x in zip(shots, x0)]

    def L(m):
        return [born(s, wav, v0[c], m[c], prec=prec).astype(f) for s, c in zip(shots, cols)]

    def LT(r):
        out = np.zeros((nx, nz), f)
        for s, c, rk in zip(shots, cols, r):
            np.add.at(out, c, born_adjoint(s, wav, v0[c], rk, prec=prec))
        return out

    def ddot(a, b):
        return float(sum(np.sum(x * y) for x, y in zip(a, b)))

    m = np.zeros((nx, nz), f)
    r = [np.asarray(d, f).copy() for d in dobs]
    rr0 = ddot(r, r)
    sg = LT(r)
    p = sg.copy()
    gamma = float(np.sum(sg * sg))
    hist = []
    for _ in range(niter):
        q = L(p)
        alpha = gamma / ddot(q, q)
        m += alpha * p
        r = [rk - alpha * qk for rk, qk in zip(r, q)]
        hist.append(ddot(r, r))
        sg = LT(r)
        gnew = float(np.sum(sg * sg))
        p = sg + (gnew / gamma) * p
        gamma = gnew
    return m, rr0, hist


def ref_set_threads(n: int):
    ref_lib().ref_set_threads(_I(n))


class RefInversion:
    """The reference's own Inversion object (src/lsrtm/inversion.cpp, compiled
    into oracle/_ref) with ns shots: sources sc [ns][2] (x, z), receivers
    gx/gz lists per shot; exposes its geometry members on flat arrays."""

    def __init__(self, sc, gxs, gzs, dx, dz, dt, fr, velfx, nx, nz, nt, delay=0, lpad=0, rpad=0):
        L = ref_lib()
        V, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.ref_inv_create.restype = V
        L.ref_inv_create.argtypes = [I, I, V, V, V, F, F, F, F, F, I, I, I, I, I, I]
        L.ref_inv_destroy.argtypes = [V]
        L.ref_inv_getvel.argtypes = [V, I, V, I, I, F, ctypes.POINTER(F), ctypes.POINTER(I), V,
                                     ctypes.c_size_t]
        L.ref_inv_getigz.argtypes = [V, F, I, I, V]
        L.ref_inv_swapreord.argtypes = [V, V, I, I, I, V, F, I, I]
        L.ref_inv_swapmodel.argtypes = [V, V, V, F, F, I, I, I, I, I]
        L.ref_inv_removedirect.argtypes = [V, V, V, I]
        self.L = L
        ns = len(gxs)
        self.ng = np.array([len(g) for g in gxs], np.int32)
        self.ngmax = int(self.ng.max())
        gc = np.zeros((ns, 2, self.ngmax), np.float32)
        for i, (gx, gz) in enumerate(zip(gxs, gzs)):
            gc[i, 0, :len(gx)] = gx
            gc[i, 1, :len(gz)] = gz
        self._sc = np.ascontiguousarray(sc, np.float32)
        self._gc = gc
        self.nt, self.nx, self.nz = nt, nx, nz
        self.h = L.ref_inv_create(ns, self.ngmax, _ptr(self.ng), _ptr(self._sc), _ptr(gc), dx, dz, dt,
                                  fr, velfx, nx, nz, nt, delay, lpad, rpad)

    def close(self):
        if self.h:
            self.L.ref_inv_destroy(self.h)
            self.h = None

    __del__ = close

    def getvel(self, is_, vel, velfx):
        vel = np.ascontiguousarray(vel, np.float32)
        nx, nz = vel.shape
        cap = 1 << 24
        out = np.zeros(cap, np.float32)
        fx, n = ctypes.c_float(), ctypes.c_int()
        rc = self.L.ref_inv_getvel(self.h, is_, _ptr(vel), nz, nx, velfx, ctypes.byref(fx),
                                   ctypes.byref(n), _ptr(out), cap)
        if rc != 0:
            raise RuntimeError("reference getVel failed")
        return fx.value, n.value, out[:n.value * nz].reshape(n.value, nz).copy()

    def getigz(self, fx_sub, nx_sub, is_):
        out = np.zeros(nx_sub, np.int32)
        if self.L.ref_inv_getigz(self.h, fx_sub, nx_sub, is_, _ptr(out)) != 0:
            raise RuntimeError("reference getIgz failed")
        return out

    def swapreord(self, csg, is_, rec, fx, adj):
        if self.L.ref_inv_swapreord(self.h, _ptr(csg), is_, csg.shape[0], csg.shape[1], _ptr(rec),
                                    fx, rec.shape[0], 1 if adj else 0) != 0:
            raise RuntimeError("reference swapReord failed")

    def swapmodel(self, m, d, mfx, dfx, add):
        if self.L.ref_inv_swapmodel(self.h, _ptr(m), _ptr(d), mfx, dfx, m.shape[1], m.shape[0],
                                    d.shape[1], d.shape[0], 1 if add else 0) != 0:
            raise RuntimeError("reference swapModel failed")

    def removedirect(self, csg, v, is_):
        if self.L.ref_inv_removedirect(self.h, _ptr(csg), _ptr(v), is_) != 0:
            raise RuntimeError("reference removeDirect failed")


_PARAM_INTS = ("nthread", "ns", "ngmax", "nx", "nz", "nt", "npml", "delay", "delaycal", "mask",
               "maxiter", "lpad", "rpad", "planeTag", "sbegin", "send")
_PARAM_FLOATS = ("dx", "dz", "dt", "fr", "velfx")
_PARAM_STRINGS = ("precsg", "wdir", "v0file", "vfile", "coordfile", "maskfile")


def ref_read_params(path):
    """The reference's Inversion::readParamFile (src/lsrtm/inversion.cpp:38-88)
    on a file: dict of the values it reads, or None where it would exit."""
    L = ref_lib()
    L.ref_param_read.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    ints = np.zeros(16, np.int32)
    floats = np.zeros(5, np.float32)
    strs = ctypes.create_string_buffer(256 * 6)
    if L.ref_param_read(path.encode(), _ptr(ints), _ptr(floats), strs) != 0:
        return None
    out = dict(zip(_PARAM_INTS, map(int, ints)))
    out.update(zip(_PARAM_FLOATS, map(np.float32, floats)))
    raw = strs.raw
    out.update((k, raw[256 * i:256 * (i + 1)].split(b"\0")[0].decode())
               for i, k in enumerate(_PARAM_STRINGS))
    return out


def ref_read_coords(path, ngmax):
    """The reference's Coords readers (src/util/coord.cpp): ns, ng, sc, gc."""
    L = ref_lib()
    L.ref_coords_count.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    L.ref_coords_read.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p]
    ns = np.zeros(1, np.int32)
    if L.ref_coords_count(path.encode(), _ptr(ns)) != 0:
        raise RuntimeError("reference countShots failed")
    ns = int(ns[0])
    ng = np.zeros(ns, np.int32)
    sc = np.zeros((ns, 2), np.float32)
    gc = np.zeros((ns, 2, ngmax), np.float32)
    if L.ref_coords_read(path.encode(), ns, ngmax, _ptr(ng), _ptr(sc), _ptr(gc)) != 0:
        raise RuntimeError("reference Coords failed")
    return ns, ng, sc, gc


def ref_plane_prepare(param_file):
    """The reference's Inversion::planeWavePrepare on a parameter file's survey."""
    L = ref_lib()
    L.ref_plane_prepare.argtypes = [ctypes.c_char_p]
    if L.ref_plane_prepare(str(param_file).encode()) != 0:
        raise RuntimeError("reference planeWavePrepare failed")


def ref_harmonic(x, kx, sx):
    """The reference's harmonic() on one trace (InitInversion.cpp:141-150)."""
    L = ref_lib()
    L.ref_harmonic.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
                               ctypes.c_float]
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros_like(x)
    if L.ref_harmonic(_ptr(x), _ptr(out), len(x), kx, sx) != 0:
        raise RuntimeError("reference harmonic failed")
    return out
