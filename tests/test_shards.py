"""Shots spread over ranks: the shard assignment, and the sharded CG loop
(seis_b200.shards.ShardedCGLS) run as two gloo ranks on CPU against the
same CGLS on one process.  The engine here is a numpy stand-in with the
phase semantics of seis_fd_lsrtm_phase_*; the GPU test drives the same loop
with the device solver."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from seis_b200.shards import ShardedCGLS, shard_shots


def test_shard_shots_balances_cost():
    rng = np.random.default_rng(0)
    costs = rng.integers(300, 738, 64) * 320
    parts = shard_shots(list(costs), 4)
    assert sorted(i for p in parts for i in p) == list(range(64))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert parts == shard_shots(list(costs), 4)  # deterministic
    assert shard_shots([5.0, 1.0], 3) == [[0], [1], []]


class NumpyEngine:
    """Linear operator A (this rank's rows) with the device solver's phases."""

    def __init__(self, A, d):
        self.A, self.d = A, d
        n = A.shape[1]
        self.s = torch.zeros(n, dtype=torch.float64)
        self.qq = torch.zeros(1, dtype=torch.float64)
        self.rr = torch.zeros(1, dtype=torch.float64)

    def phase_reset(self, s, rr):
        self.m = np.zeros(self.A.shape[1])
        self.r = self.d.copy()
        rr[0] = float(self.r @ self.r)
        s[:] = torch.from_numpy(self.A.T @ self.r)

    def phase_direction(self, s, first):
        sv = s.numpy()
        g = float(sv @ sv)
        if first:
            self.gamma, self.p = g, sv.copy()
        else:
            beta, self.gamma = g / self.gamma, g
            self.p = sv + beta * self.p

    def phase_forward(self, qq):
        self.q = self.A @ self.p
        qq[0] = float(self.q @ self.q)

    def phase_update(self, qq, s, rr):
        alpha = self.gamma / float(qq[0])
        self.m = self.m + alpha * self.p
        self.r = self.r - alpha * self.q
        rr[0] = float(self.r @ self.r)
        s[:] = torch.from_numpy(self.A.T @ self.r)

    def read_rr(self):
        return float(self.rr[0])


def problem(seed=3, rows=(40, 25), n=30):
    rng = np.random.default_rng(seed)
    A = [rng.standard_normal((k, n)) for k in rows]
    d = [rng.standard_normal(k) for k in rows]
    return A, d


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A, d = problem()
        eng = NumpyEngine(A[rank], d[rank])
        cg = ShardedCGLS(eng, lambda b: dist.all_reduce(b))
        hist = [cg.reset()] + cg.iterate(6)
        out.put((rank, hist, eng.m))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_cgls_two_gloo_ranks_match_one_process():
    A, d = problem()
    one = NumpyEngine(np.vstack(A), np.concatenate(d))
    cg = ShardedCGLS(one, lambda b: None)
    want = [cg.reset()] + cg.iterate(6)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for rank, hist, m in res:
        np.testing.assert_allclose(hist, want, rtol=1e-10)
        np.testing.assert_allclose(m, one.m, rtol=1e-9, atol=1e-12)
    assert np.all(np.diff(want) < 0)
