"""The sharded LSRTM loop (seis_b200.shards.ShardedCGLS) over the device
solver's phases (seis_fd_lsrtm_phase_*): two processes, each with half of a
small survey's shots on its own context, sum the image and the FP64 scalars
through a gloo group (host copies), and must follow the single-process
solver over all shots.  The processes share one GPU; their kernels never wait
on one another (the only exchange is the host-side all-reduce between
phases).  The per-rank partial images are summed in another order than the
single process's shot loop, so agreement is to FP32 rounding, not bitwise."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NZ, NT = 160, 60, 300


def survey():
    from seis_b200 import Shot
    rng = np.random.default_rng(11)
    v = np.repeat(np.sort(rng.uniform(1800, 3200, 6)), NZ // 6)[None, :].repeat(NX, 0)
    v = v.astype(np.float32)
    v0 = v.copy()
    for _ in range(3):  # smooth background
        v0 = (v0 + np.roll(v0, 1, 1) + np.roll(v0, -1, 1)) / 3
    v0[:, 0], v0[:, -1] = v[:, 0], v[:, -1]
    shots, x0 = [], []
    for nx_s, x in ((90, 0), (120, 40), (70, 90), (100, 60)):
        shots.append(Shot(nx=nx_s, nz=NZ, pml=12, nt=NT, ndel=40, sx=nx_s // 2, sz=1, dt=1e-3,
                          dx=10.0, dz=10.0, gz=np.ones(nx_s, np.int32)))
        x0.append(x)
    return v, v0.astype(np.float32), shots, x0


def observed(ctx, v, v0, shots, x0, wav):
    from seis_b200._lib import IN_DV, IN_VEL, IN_WAVELET, OP_BORN, OUT_GATHER, Plan
    dv = v - v0
    with Plan(ctx, OP_BORN, shots) as p:
        for i, (s, x) in enumerate(zip(shots, x0)):
            p.set(i, IN_VEL, np.ascontiguousarray(v0[x:x + s.nx]))
            p.set(i, IN_DV, np.ascontiguousarray(dv[x:x + s.nx]))
            p.set(i, IN_WAVELET, wav)
        p.run()
        return [p.get(i, OUT_GATHER) for i in range(len(shots))]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        from seis_b200 import Context
        from seis_b200._lib import SNAP_BF16, Lsrtm, ricker
        from seis_b200.shards import DeviceEngine, ShardedCGLS, host_reduce
        torch.cuda.set_device(0)
        v, v0, shots, x0 = survey()
        wav = ricker(1e-3, 25.0, 40, NT + 40)
        mine = [0, 1] if rank == 0 else [2, 3]
        with Context(0) as ctx:
            d = observed(ctx, v, v0, shots, x0, wav)
            with Lsrtm(ctx, NX, NZ, [shots[i] for i in mine], [x0[i] for i in mine],
                       snap_every=2, snap_dtype=SNAP_BF16) as ls:
                ls.set_background(v0, wav)
                for k, i in enumerate(mine):
                    ls.set_data(k, d[i])
                eng = DeviceEngine(ls)
                cg = ShardedCGLS(eng, host_reduce(eng))
                hist = [cg.reset()] + cg.iterate(3)
                q.put((rank, hist, ls.model()))
    except Exception as e:  # reported to the parent, never left hanging
        q.put((rank, repr(e), None))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_processes_follow_one(ctx):
    import torch.multiprocessing as mp

    from seis_b200._lib import SNAP_BF16, Lsrtm, ricker
    v, v0, shots, x0 = survey()
    wav = ricker(1e-3, 25.0, 40, NT + 40)
    d = observed(ctx, v, v0, shots, x0, wav)
    with Lsrtm(ctx, NX, NZ, shots, x0, snap_every=2, snap_dtype=SNAP_BF16) as ls:
        ls.set_background(v0, wav)
        for i in range(len(shots)):
            ls.set_data(i, d[i])
        want = [ls.reset()] + list(ls.iterate(3))
        m_want = ls.model()
    mpc = mp.get_context("spawn")
    q = mpc.Queue()
    port = free_port()
    procs = [mpc.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = [q.get(timeout=300) for _ in procs]
    finally:
        for p in procs:
            p.join(120)
    for p in procs:
        assert p.exitcode == 0
    for rank, hist, m in res:
        assert m is not None, hist
        err_h = np.max(np.abs(np.array(hist) - want) / np.array(want))
        err_m = float(np.linalg.norm(m - m_want) / np.linalg.norm(m_want))
        print(f"rank {rank}: residual history rel {err_h:.2e}, model rel L2 {err_m:.2e}")
        assert err_h <= 1e-5 and err_m <= 1e-5
    assert np.all(np.diff(want) < 0)
