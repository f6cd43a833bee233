"""The shot driver (include/seis_driver.h): the reference's parameter file,
coordinate file and per-shot gather files driving the batched engine.

It stands where the reference's MPI driver class ``Inversion``
(src/lsrtm/inversion.cpp) stands: ``readParamFile`` / ``getConfig`` read the
same files with the same rules, and ``modeling``, ``born``, ``rtm`` follow
``modeling_MPI``, ``forward_MPI`` and ``adjoint_MPI`` shot for shot, writing
the same file names and raw float32 layouts; ``lsrtm`` is the CG solver the
reference declares (``cgsolver_MPI``) but does not define.

    python -m seis_b200.driver PARAM_FILE
        {modeling|born|rtm|lsrtm|illum|plane_prepare|rtm_plane|illum_plane} [options]
"""
from __future__ import annotations

import argparse
import ctypes
import sys

import numpy as np

from ._lib import Context, LsrtmOptsC, SNAP_F16, SeisError, lib

_P, _I = ctypes.c_void_p, ctypes.c_int


class Params(ctypes.Structure):
    """seis_params: the reference's paramLSRTM values (src/lsrtm/datastr.h)."""
    _fields_ = [(n, ctypes.c_int) for n in (
        "nthread", "ns", "ngmax", "nx", "nz", "nt", "npml", "delay", "delaycal", "mask", "maxiter",
        "lpad", "rpad", "planeTag", "sbegin", "send")] + \
        [(n, ctypes.c_float) for n in ("dx", "dz", "dt", "fr", "velfx")] + \
        [("np", ctypes.c_int), ("dp", ctypes.c_float), ("pmin", ctypes.c_float)] + \
        [(n, ctypes.c_char * 256) for n in ("precsg", "wdir", "v0file", "vfile", "coordfile",
                                            "maskfile")]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = v.decode() if isinstance(v, bytes) else v
        return out


def _setup():
    L = lib()
    if getattr(L, "_driver_ready", False):
        return L
    L.seis_params_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(Params), ctypes.c_char_p,
                                   ctypes.c_size_t]
    L.seis_coords_count.argtypes = [ctypes.c_char_p, ctypes.POINTER(_I)]
    L.seis_coords_read.argtypes = [ctypes.c_char_p, _I, _I, _P, _P, _P]
    L.seis_driver_create.argtypes = [_P, ctypes.c_char_p, _I, ctypes.POINTER(_P)]
    L.seis_driver_destroy.argtypes = [_P]
    L.seis_driver_params.argtypes = [_P]
    L.seis_driver_params.restype = ctypes.POINTER(Params)
    L.seis_driver_modeling.argtypes = [_P, _P]
    L.seis_driver_born.argtypes = [_P, _P]
    L.seis_driver_rtm.argtypes = [_P, _I, _P]
    L.seis_driver_illum.argtypes = [_P, _P]
    L.seis_driver_plane_prepare.argtypes = [_P]
    L.seis_driver_rtm_plane.argtypes = [_P, _I, _P]
    L.seis_driver_illum_plane.argtypes = [_P, _P]
    L.seis_driver_lsrtm.argtypes = [_P, _I, _I, ctypes.POINTER(LsrtmOptsC), _P, _P]
    L._driver_ready = True
    return L


def read_params(path: str) -> Params:
    """Parameter file with the reference parser's rules (Inversion::readParamFile)."""
    L = _setup()
    p = Params()
    err = ctypes.create_string_buffer(512)
    rc = L.seis_params_read(path.encode(), ctypes.byref(p), err, len(err))
    if rc:
        raise SeisError(f"{path}: {err.value.decode()}")
    return p


def read_coords(path: str, ngmax: int = None):
    """(ng [ns], sc [ns][2], gc [ns][2][ngmax]) of a coordinate file (Coords)."""
    L = _setup()
    ns = _I()
    if L.seis_coords_count(path.encode(), ctypes.byref(ns)):
        raise SeisError(f"{path}: cannot read")
    ns = ns.value
    if ngmax is None:  # a first pass finds the largest shot
        ng = np.zeros(ns, np.int32)
        big = 1 << 16
        sc = np.zeros((ns, 2), np.float32)
        gc = np.zeros((ns, 2, big), np.float32)
        if L.seis_coords_read(path.encode(), ns, big, ng.ctypes.data, sc.ctypes.data,
                              gc.ctypes.data):
            raise SeisError(f"{path}: cannot read")
        ngmax = max(int(ng.max()), 1)
    ng = np.zeros(ns, np.int32)
    sc = np.zeros((ns, 2), np.float32)
    gc = np.zeros((ns, 2, ngmax), np.float32)
    if L.seis_coords_read(path.encode(), ns, ngmax, ng.ctypes.data, sc.ctypes.data, gc.ctypes.data):
        raise SeisError(f"{path}: cannot read")
    return ng, sc, gc


class Driver:
    """A parameter file's survey on one device context."""

    def __init__(self, ctx, param_file: str, batch: int = 0):
        """ctx: a Context, or None for the host-only steps (plane_prepare)."""
        self.ctx = ctx
        self.L = _setup()
        h = _P()
        rc = self.L.seis_driver_create(ctx.h if ctx is not None else None, param_file.encode(),
                                       batch, ctypes.byref(h))
        if rc:
            raise SeisError(f"{param_file}: driver setup failed ({rc})")
        self.h = h
        # a copy: it outlives the driver
        self.params = Params.from_buffer_copy(self.L.seis_driver_params(h).contents)

    def _run(self, rc, what):
        if rc:
            msg = self.ctx.L.seis_fd_last_error(self.ctx.h) if self.ctx is not None else b""
            raise SeisError(f"{what} failed ({rc}): {msg}")

    def plane_prepare(self):
        """Phase-encoded sources and data PLANE_S_NEW<k>.dat / PLANE_R_NEW<k>.dat
        (planeWavePrepare); host only."""
        self._run(self.L.seis_driver_plane_prepare(self.h), "plane_prepare")

    def modeling(self, v: np.ndarray = None):
        """Synthetic gathers precsg<is>.dat of v [nx][nz] (None: the vfile model)."""
        a = None if v is None else np.ascontiguousarray(v, np.float32)
        self._run(self.L.seis_driver_modeling(self.h, None if a is None else a.ctypes.data),
                  "modeling")

    def born(self, dv: np.ndarray):
        """Born gathers wdir BORN<is>.dat of the perturbation dv [nx][nz]."""
        a = np.ascontiguousarray(dv, np.float32)
        self._run(self.L.seis_driver_born(self.h, a.ctypes.data), "born")

    def rtm(self, born_data: bool = False) -> np.ndarray:
        """Reference RTM image [nx][nz] of shots sbegin..send."""
        img = np.zeros((self.params.nx, self.params.nz), np.float32)
        self._run(self.L.seis_driver_rtm(self.h, 1 if born_data else 0, img.ctypes.data), "rtm")
        return img

    def rtm_plane(self, born_data: bool = False) -> np.ndarray:
        """Plane-wave RTM image [nx][nz] summed over the np wavenumbers (adjointPlane_MPI)."""
        img = np.zeros((self.params.nx, self.params.nz), np.float32)
        self._run(self.L.seis_driver_rtm_plane(self.h, 1 if born_data else 0, img.ctypes.data),
                  "rtm_plane")
        return img

    def illum_plane(self) -> np.ndarray:
        """Plane-wave illumination [nx][nz] summed over the np wavenumbers; each one
        is also written to wdir ILLUM_PLANE<k>.dat (illumPlane_MPI)."""
        ss = np.zeros((self.params.nx, self.params.nz), np.float32)
        self._run(self.L.seis_driver_illum_plane(self.h, ss.ctypes.data), "illum_plane")
        return ss

    def illum(self) -> np.ndarray:
        """Source illumination [nx][nz] of all shots (illum_MPI)."""
        ss = np.zeros((self.params.nx, self.params.nz), np.float32)
        self._run(self.L.seis_driver_illum(self.h, ss.ctypes.data), "illum")
        return ss

    def lsrtm(self, niter: int, born_data: bool = False, snap_every: int = 1,
              snap_dtype: int = SNAP_F16, exact: bool = False, checkpoint_every: int = 0,
              group_shots: int = 0):
        """(model [nx][nz], [|d|^2, |r|^2 per iteration]) of CGLS over all shots;
        checkpoint_every > 0 keeps source-field checkpoints instead of every snapshot,
        group_shots > 0 builds the plans of that many shots at a time."""
        img = np.zeros((self.params.nx, self.params.nz), np.float32)
        rr = np.zeros(niter + 1, np.float64)
        o = LsrtmOptsC(snap_every, snap_dtype, 1 if exact else 0, checkpoint_every, group_shots)
        self._run(self.L.seis_driver_lsrtm(self.h, 1 if born_data else 0, niter, ctypes.byref(o),
                                           img.ctypes.data, rr.ctypes.data), "lsrtm")
        return img, rr

    def close(self):
        if getattr(self, "h", None):
            self.L.seis_driver_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m seis_b200.driver", description=__doc__.split("\n")[0])
    ap.add_argument("param_file")
    ap.add_argument("op", choices=["modeling", "born", "rtm", "lsrtm", "illum", "plane_prepare",
                                   "rtm_plane", "illum_plane"])
    ap.add_argument("--dv", help="perturbation [nx][nz] float32 file (born)")
    ap.add_argument("--born-data", action="store_true", help="rtm/lsrtm from BORN<is>.dat")
    ap.add_argument("--niter", type=int, default=None, help="lsrtm iterations (default maxiter)")
    ap.add_argument("--out", help="image file (rtm, lsrtm)")
    ap.add_argument("--batch", type=int, default=0, help="shots per device batch (0: all)")
    ap.add_argument("--checkpoint-every", type=int, default=0,
                    help="lsrtm: source-field checkpoint interval (0: keep every snapshot)")
    ap.add_argument("--group-shots", type=int, default=0,
                    help="lsrtm: shots whose plans are built at a time (0: all)")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    if a.op == "plane_prepare":
        with Driver(None, a.param_file) as d:
            d.plane_prepare()
        return 0
    with Context(a.device) as ctx, Driver(ctx, a.param_file, a.batch) as d:
        p = d.params
        if a.op == "modeling":
            d.modeling()
        elif a.op == "born":
            d.born(np.fromfile(a.dv, np.float32).reshape(p.nx, p.nz))
        else:
            if a.op == "rtm":
                img = d.rtm(a.born_data)
            elif a.op == "illum":
                img = d.illum()
            elif a.op == "rtm_plane":
                img = d.rtm_plane(a.born_data)
            elif a.op == "illum_plane":
                img = d.illum_plane()
            else:
                img, rr = d.lsrtm(a.niter if a.niter is not None else p.maxiter, a.born_data,
                                  checkpoint_every=a.checkpoint_every,
                                  group_shots=a.group_shots)
                for i, r in enumerate(rr):
                    print(f"iteration {i}: |r|^2 = {r:.6e}")
            if a.out:
                img.tofile(a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
