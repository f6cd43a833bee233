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
        return shot_desc(self)


def shot_desc(s) -> ShotDescC:
    """``seis_shot_desc`` of any record with the fields of ``Shot`` (this
    class, or the survey records of ``seis_b200.synth``)."""
    gz = np.ascontiguousarray(s.gz, np.int32)
    d = ShotDescC(int(s.nx), int(s.nz), int(s.pml), int(s.nt), int(s.ndel), int(s.sx), int(s.sz),
                  float(s.dt), float(s.dx), float(s.dz),
                  gz.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    d._keep = gz  # keep the receiver array alive with the struct
    return d


class LsrtmOptsC(ctypes.Structure):
    _fields_ = [("snap_every", ctypes.c_int), ("snap_dtype", ctypes.c_int),
                ("exact", ctypes.c_int), ("checkpoint_every", ctypes.c_int),
                ("group_shots", ctypes.c_int), ("tile_shape", ctypes.c_int)]


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
        L.seis_fd_stream.argtypes = [P]
        L.seis_fd_stream.restype = P
        L.seis_fd_ricker.argtypes = [ctypes.c_float, ctypes.c_float, I, I, P]
        L.seis_fd_validate_shot.argtypes = [SD, ctypes.c_char_p, ctypes.c_size_t]
        L.seis_fd_modeling.argtypes = [P, SD, P, P, P]
        L.seis_fd_plan_create.argtypes = [P, I, I, SD, ctypes.POINTER(P)]
        L.seis_fd_plan_destroy.argtypes = [P]
        L.seis_fd_plan_set.argtypes = [P, I, I, P]
        L.seis_fd_plan_set_device.argtypes = [P, I, I, P]
        L.seis_fd_plan_run.argtypes = [P]
        L.seis_fd_plan_get.argtypes = [P, I, I, P]
        L.seis_fd_plan_sync.argtypes = [P]
        L.seis_fd_plan_cell_updates.argtypes = [P]
        L.seis_fd_plan_cell_updates.restype = ctypes.c_int64
        L.seis_fd_plan_launches_per_run.argtypes = [P]
        L.seis_fd_plan_launches_per_run.restype = ctypes.c_int64
        L.seis_fd_plan_set_exact.argtypes = [P, I]
        L.seis_fd_plan_set_snapshots.argtypes = [P, I, I]
        L.seis_fd_plan_set_checkpoints.argtypes = [P, I]
        L.seis_fd_plan_device_bytes.argtypes = [P]
        L.seis_fd_plan_device_bytes.restype = ctypes.c_int64
        L.seis_fd_born_adjoint.argtypes = [P, SD, P, P, P, P]
        L.seis_fd_plan_time_kernels.argtypes = [P, I, ctypes.POINTER(ctypes.c_double),
                                                ctypes.POINTER(ctypes.c_double)]
        L.seis_fd_plan_set_tile_shape.argtypes = [P, I]
        L.seis_fd_plan_tile_shape.argtypes = [P]
        L.seis_fd_plan_set_launch.argtypes = [P, I]
        L.seis_fd_plan_launch.argtypes = [P]
        L.seis_fd_plan_autotune.argtypes = [P, I, I, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_int)]
        PP = ctypes.POINTER(P)
        L.seis_fd_modeling_batch.argtypes = [P, I, SD, PP, PP, PP]
        L.seis_fd_born_batch.argtypes = [P, I, SD, PP, PP, PP, PP]
        L.seis_fd_rtm_batch.argtypes = [P, I, SD, PP, PP, PP, PP]
        L.seis_fd_born.argtypes = [P, SD, P, P, P, P]
        L.seis_fd_rtm.argtypes = [P, SD, P, P, P, P]
        L.seis_fd_illum.argtypes = [P, SD, P, P, P]
        L.seis_fd_born_plane.argtypes = [P, SD, P, P, P, P]
        L.seis_fd_rtm_plane.argtypes = [P, SD, P, P, P, P]
        L.seis_fd_rtm_true.argtypes = [P, SD, P, P, P, P]
        L.seis_fd_rtm_updown.argtypes = [P, SD, P, P, P, P, P, P]
        L.seis_fd_illum_plane.argtypes = [P, SD, P, P, P]
        L.seis_fd_hilbert.argtypes = [P, P, I, I]
        L.seis_fd_illum_batch.argtypes = [P, I, SD, PP, PP, PP]
        L.seis_fd_vec_dot.argtypes = [P, P, P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)]
        L.seis_fd_vec_axpby.argtypes = [P, P, P, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_size_t]
        L.seis_fd_lsrtm_create.argtypes = [P, I, I, I, SD, ctypes.POINTER(I),
                                           ctypes.POINTER(LsrtmOptsC), PP]
        L.seis_fd_lsrtm_destroy.argtypes = [P]
        L.seis_fd_lsrtm_create_mapped.argtypes = [P, I, I, I, SD, ctypes.POINTER(I),
                                                  ctypes.POINTER(LsrtmOptsC), PP]
        L.seis_fd_lsrtm_phase_reset.argtypes = [P, P, P]
        L.seis_fd_lsrtm_phase_forward.argtypes = [P, P]
        L.seis_fd_lsrtm_phase_update.argtypes = [P, P, P, P]
        L.seis_fd_lsrtm_phase_direction.argtypes = [P, P, I]
        L.seis_fd_lsrtm_set_background.argtypes = [P, P, P]
        L.seis_fd_lsrtm_set_data.argtypes = [P, I, P]
        L.seis_fd_lsrtm_reset.argtypes = [P, P]
        L.seis_fd_lsrtm_iterate.argtypes = [P, I, P]
        L.seis_fd_lsrtm_model.argtypes = [P, P]
        L.seis_fd_lsrtm_cell_updates.argtypes = [P]
        L.seis_fd_lsrtm_cell_updates.restype = ctypes.c_int64
        L.seis_fd_lsrtm_device_bytes.argtypes = [P]
        L.seis_fd_lsrtm_device_bytes.restype = ctypes.c_int64
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
    def stream_ptr(self) -> int:
        """cudaStream_t of this context (as an integer)."""
        return int(self.L.seis_fd_stream(self.h) or 0)

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
    rc = lib().seis_fd_validate_shot(shot_desc(shot), buf, 512)
    return "" if rc == SEIS_OK else (buf.value.decode() or f"error {rc}")


(OP_MODELING, OP_BORN, OP_RTM, OP_BORN_ADJOINT, OP_ILLUM, OP_BORN_PLANE, OP_RTM_PLANE,
 OP_RTM_TRUE, OP_RTM_UPDOWN, OP_ILLUM_PLANE) = range(10)
SNAP_F32, SNAP_BF16, SNAP_F16 = 1, 2, 3
# tile shapes of the step kernels (include/seis_fd.h SEIS_TILE_*)
LAUNCH_OVERLAP, LAUNCH_PERSISTENT, LAUNCH_PER_TILE = 1, 2, 4  # include/seis_fd.h SEIS_LAUNCH_*
TILE_32x64, TILE_64x32, TILE_16x128, TILE_64x64, TILE_32x32 = range(5)
TILE_SHAPES = {TILE_32x64: (32, 64), TILE_64x32: (64, 32), TILE_16x128: (16, 128),
               TILE_64x64: (64, 64), TILE_32x32: (32, 32)}
IN_VEL, IN_DV, IN_WAVELET, IN_GATHER, IN_SOURCE, IN_WAVELET_H = 0, 1, 2, 3, 4, 5
OUT_GATHER, OUT_IMAGE, OUT_COMPONENTS = 0, 1, 2


def shot_array(shots):
    arr = (ShotDescC * len(shots))()
    keep = []
    for i, s in enumerate(shots):
        c = shot_desc(s)
        keep.append(c._keep)
        arr[i] = c
    arr._keep = keep
    return arr


class Plan:
    """A batch of shots resident on the device (seis_fd_plan_*)."""

    def __init__(self, ctx: Context, op: int, shots):
        self.ctx, self.op, self.shots = ctx, op, list(shots)
        self._descs = shot_array(self.shots)
        h = ctypes.c_void_p()
        ctx.check(ctx.L.seis_fd_plan_create(ctx.h, op, len(self.shots), self._descs, ctypes.byref(h)))
        self.h = h

    def set(self, shot: int, what: int, arr: np.ndarray):
        a = np.ascontiguousarray(arr, np.float32)
        self.ctx.check(self.ctx.L.seis_fd_plan_set(self.h, shot, what, ptr(a)))
        self.ctx.check(self.ctx.L.seis_fd_plan_sync(self.h))

    def set_device(self, shot: int, what: int, dev_ptr: int):
        self.ctx.check(self.ctx.L.seis_fd_plan_set_device(self.h, shot, what, ctypes.c_void_p(dev_ptr)))

    def run(self):
        self.ctx.check(self.ctx.L.seis_fd_plan_run(self.h))

    def sync(self):
        self.ctx.check(self.ctx.L.seis_fd_plan_sync(self.h))

    def get(self, shot: int, what: int, out: np.ndarray = None) -> np.ndarray:
        s = self.shots[shot]
        shape = (s.nx, s.nt) if what == OUT_GATHER else (s.nx, s.nz)
        if out is None:
            out = np.zeros(shape, np.float32)
        self.ctx.check(self.ctx.L.seis_fd_plan_get(self.h, shot, what, ptr(out)))
        return out

    def set_snapshots(self, every: int = 1, dtype: int = 1):
        self.ctx.check(self.ctx.L.seis_fd_plan_set_snapshots(self.h, every, dtype))

    def set_checkpoints(self, every: int):
        """Keep source-field checkpoints every `every` steps instead of every
        snapshot (seis_fd_plan_set_checkpoints); 0 = keep every snapshot."""
        self.ctx.check(self.ctx.L.seis_fd_plan_set_checkpoints(self.h, every))

    @property
    def device_bytes(self) -> int:
        return int(self.ctx.L.seis_fd_plan_device_bytes(self.h))

    def set_exact(self, exact: bool):
        self.ctx.check(self.ctx.L.seis_fd_plan_set_exact(self.h, 1 if exact else 0))

    def set_tile_shape(self, shape: int):
        self.ctx.check(self.ctx.L.seis_fd_plan_set_tile_shape(self.h, shape))

    @property
    def tile_shape(self) -> int:
        return int(self.ctx.L.seis_fd_plan_tile_shape(self.h))

    def set_launch(self, flags: int):
        """LAUNCH_* flags (include/seis_fd.h): overlap the interior and pad
        kernels of a step; persistent or one-tile-per-CTA interior kernel."""
        self.ctx.check(self.ctx.L.seis_fd_plan_set_launch(self.h, flags))

    @property
    def launch(self) -> int:
        return int(self.ctx.L.seis_fd_plan_launch(self.h))

    def autotune(self, steps: int = 10, force: bool = False):
        """(chosen shape, shortest mean step ms of every shape over the launch
        forms; 0 where not timed).  The launch form kept is `launch`."""
        ms = (ctypes.c_double * len(TILE_SHAPES))()
        best = ctypes.c_int()
        self.ctx.check(self.ctx.L.seis_fd_plan_autotune(self.h, steps, 1 if force else 0, ms,
                                                        ctypes.byref(best)))
        return best.value, list(ms)

    def time_kernels(self, steps: int):
        ms = (ctypes.c_double * 3)()
        by = (ctypes.c_double * 2)()
        self.ctx.check(self.ctx.L.seis_fd_plan_time_kernels(self.h, steps, ms, by))
        return list(ms), list(by)

    @property
    def cell_updates(self) -> int:
        return int(self.ctx.L.seis_fd_plan_cell_updates(self.h))

    @property
    def launches_per_run(self) -> int:
        return int(self.ctx.L.seis_fd_plan_launches_per_run(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.seis_fd_plan_destroy(self.h)
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


def _ptr_list(arrays):
    lst = (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    return lst


def batch(ctx: Context, op: int, shots, wavs, vels, third=None):
    """One-call batched operator (seis_fd_*_batch); returns per-shot outputs."""
    shots = list(shots)
    descs = shot_array(shots)
    wavs = [np.ascontiguousarray(w, np.float32) for w in wavs]
    vels = [np.ascontiguousarray(v, np.float32) for v in vels]
    if op in (OP_RTM, OP_ILLUM):
        outs = [np.zeros((s.nx, s.nz), np.float32) for s in shots]
    else:
        outs = [np.zeros((s.nx, s.nt), np.float32) for s in shots]
    pw, pv, po = _ptr_list(wavs), _ptr_list(vels), _ptr_list(outs)
    n = len(shots)
    if op == OP_ILLUM:
        rc = ctx.L.seis_fd_illum_batch(ctx.h, n, descs, pw, pv, po)
    elif op == OP_MODELING:
        rc = ctx.L.seis_fd_modeling_batch(ctx.h, n, descs, pw, pv, po)
    else:
        thirds = [np.ascontiguousarray(t, np.float32) for t in third]
        pt = _ptr_list(thirds)
        fn = ctx.L.seis_fd_born_batch if op == OP_BORN else ctx.L.seis_fd_rtm_batch
        rc = fn(ctx.h, n, descs, pw, pv, pt, po)
    ctx.check(rc)
    return outs


class Lsrtm:
    """Least-squares RTM by CGLS on a global nx x nz grid (seis_fd_lsrtm_*).

    Shot k covers columns x0[k] .. x0[k] + shots[k].nx - 1 of the model.
    """

    def __init__(self, ctx: Context, nx: int, nz: int, shots, x0=None, snap_every: int = 1,
                 snap_dtype: int = None, exact: bool = False, colmaps=None,
                 checkpoint_every: int = 0, group_shots: int = 0, tile_shape: int = None):
        """Shot k covers columns x0[k] .. x0[k] + nx_k - 1, or the model columns
        colmaps[k] (one per sub-grid column, non-decreasing).  checkpoint_every > 0
        keeps source-field checkpoints instead of every snapshot; group_shots > 0
        builds the plans of that many shots at a time in every operator
        application instead of keeping all of them.  tile_shape: None (default)
        lets the autotuner pick each plan's tile shape; else a TILE_* shape."""
        self.ctx, self.nx, self.nz, self.shots = ctx, nx, nz, list(shots)
        self._descs = shot_array(self.shots)
        o = LsrtmOptsC(snap_every, SNAP_F16 if snap_dtype is None else snap_dtype,
                       1 if exact else 0, checkpoint_every, group_shots,
                       0 if tile_shape is None else tile_shape + 1)
        h = ctypes.c_void_p()
        if colmaps is None:
            self._x0 = (ctypes.c_int * len(self.shots))(*[int(v) for v in x0])
            ctx.check(ctx.L.seis_fd_lsrtm_create(ctx.h, nx, nz, len(self.shots), self._descs,
                                                 self._x0, ctypes.byref(o), ctypes.byref(h)))
        else:
            flat = np.concatenate([np.asarray(c, np.int32) for c in colmaps])
            self._map = (ctypes.c_int * len(flat))(*[int(v) for v in flat])
            ctx.check(ctx.L.seis_fd_lsrtm_create_mapped(ctx.h, nx, nz, len(self.shots),
                                                        self._descs, self._map, ctypes.byref(o),
                                                        ctypes.byref(h)))
        self.h = h

    # phases of one iteration on device buffers (pointers as integers), for
    # solvers spread over several devices; see include/seis_fd.h
    def phase_reset(self, d_s: int, d_rr: int):
        self.ctx.check(self.ctx.L.seis_fd_lsrtm_phase_reset(self.h, d_s, d_rr))

    def phase_forward(self, d_qq: int):
        self.ctx.check(self.ctx.L.seis_fd_lsrtm_phase_forward(self.h, d_qq))

    def phase_update(self, d_qq: int, d_s: int, d_rr: int):
        self.ctx.check(self.ctx.L.seis_fd_lsrtm_phase_update(self.h, d_qq, d_s, d_rr))

    def phase_direction(self, d_s: int, first: bool):
        self.ctx.check(self.ctx.L.seis_fd_lsrtm_phase_direction(self.h, d_s, 1 if first else 0))

    def set_background(self, v0: np.ndarray, wav: np.ndarray):
        v = np.ascontiguousarray(v0, np.float32)
        w = np.ascontiguousarray(wav, np.float32)
        assert v.shape == (self.nx, self.nz)
        self.ctx.check(self.ctx.L.seis_fd_lsrtm_set_background(self.h, ptr(v), ptr(w)))

    def set_data(self, shot: int, d: np.ndarray):
        a = np.ascontiguousarray(d, np.float32)
        s = self.shots[shot]
        assert a.shape == (s.nx, s.nt)
        self.ctx.check(self.ctx.L.seis_fd_lsrtm_set_data(self.h, shot, ptr(a)))

    def reset(self) -> float:
        rr = ctypes.c_double()
        self.ctx.check(self.ctx.L.seis_fd_lsrtm_reset(self.h, ctypes.byref(rr)))
        return rr.value

    def iterate(self, niter: int = 1) -> np.ndarray:
        rr = np.zeros(niter, np.float64)
        self.ctx.check(self.ctx.L.seis_fd_lsrtm_iterate(self.h, niter, ptr(rr)))
        return rr

    def model(self) -> np.ndarray:
        m = np.zeros((self.nx, self.nz), np.float32)
        self.ctx.check(self.ctx.L.seis_fd_lsrtm_model(self.h, ptr(m)))
        return m

    @property
    def cell_updates(self) -> int:
        return int(self.ctx.L.seis_fd_lsrtm_cell_updates(self.h))

    @property
    def device_bytes(self) -> int:
        return int(self.ctx.L.seis_fd_lsrtm_device_bytes(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.seis_fd_lsrtm_destroy(self.h)
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


def vec_dot(ctx: Context, a_ptr: int, b_ptr: int, n: int) -> float:
    out = ctypes.c_double()
    ctx.check(ctx.L.seis_fd_vec_dot(ctx.h, ctypes.c_void_p(a_ptr), ctypes.c_void_p(b_ptr), n,
                                    ctypes.byref(out)))
    return out.value


def vec_axpby(ctx: Context, y_ptr: int, x_ptr: int, a: float, b: float, n: int):
    ctx.check(ctx.L.seis_fd_vec_axpby(ctx.h, ctypes.c_void_p(y_ptr), ctypes.c_void_p(x_ptr),
                                      a, b, n))
