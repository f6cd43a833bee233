"""Shots spread over several devices: one process per GPU, each with its own
shots, the same model grid and the same CG state.

The reference farms shots to MPI workers and sums their per-shot images
through files (Inversion::masterRun / adjoint_MPI, src/lsrtm/inversion.cpp:
365-474, :753-807).  Here each rank runs its shard as one batch, and a CG
iteration exchanges, in place on the device, exactly what the solver needs
summed: |q|^2 after the forward operator, then the image L^T r and |r|^2.
`ShardedCGLS` is that loop over any engine with the four phases of
seis_fd_lsrtm_phase_* and a `reduce(buffer)` that sums a buffer over the ranks
(torch.distributed.all_reduce on the engine's stream for NCCL; the CPU tests
use gloo with a numpy engine).
"""
from __future__ import annotations

from typing import Callable, List, Sequence


def shard_shots(costs: Sequence[float], world: int) -> List[List[int]]:
    """Shots per rank, balancing the summed cost (largest first onto the
    least loaded rank; ties to the lower rank); each rank's list is sorted."""
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda j: (load[j], j))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in out]


class ShardedCGLS:
    """CGLS with the shots split over ranks (see module docstring).

    engine: phase_reset(s, rr), phase_forward(qq), phase_update(qq, s, rr),
    phase_direction(s, first) on its buffers `s`, `qq`, `rr`; sync();
    read_rr() -> float.  reduce(buf): in-place sum over the ranks."""

    def __init__(self, engine, reduce: Callable):
        self.e, self.reduce = engine, reduce

    def reset(self) -> float:
        e = self.e
        e.phase_reset(e.s, e.rr)
        self.reduce(e.s)
        self.reduce(e.rr)
        e.phase_direction(e.s, True)
        return e.read_rr()

    def iterate(self, niter: int) -> List[float]:
        e, out = self.e, []
        for _ in range(niter):
            e.phase_forward(e.qq)
            self.reduce(e.qq)
            e.phase_update(e.qq, e.s, e.rr)
            self.reduce(e.s)
            self.reduce(e.rr)
            e.phase_direction(e.s, False)
            out.append(e.read_rr())
        return out


class DeviceEngine:
    """The phases of a seis_b200 Lsrtm solver on torch device buffers (the
    buffers torch.distributed reduces), all ordered on the solver's stream."""

    def __init__(self, ls):
        import torch
        self.ls = ls
        dev = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.ExternalStream(ls.ctx.stream_ptr, device=dev)
        self.s = torch.zeros((ls.nx, ls.nz), dtype=torch.float32, device=dev)
        self.qq = torch.zeros(1, dtype=torch.float64, device=dev)
        self.rr = torch.zeros(1, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()

    def phase_reset(self, s, rr):
        self.ls.phase_reset(s.data_ptr(), rr.data_ptr())

    def phase_forward(self, qq):
        self.ls.phase_forward(qq.data_ptr())

    def phase_update(self, qq, s, rr):
        self.ls.phase_update(qq.data_ptr(), s.data_ptr(), rr.data_ptr())

    def phase_direction(self, s, first):
        self.ls.phase_direction(s.data_ptr(), first)

    def read_rr(self) -> float:
        import torch
        with torch.cuda.stream(self.stream):
            v = float(self.rr.item())  # synchronises the solver's stream
        return v


def nccl_reduce(engine: DeviceEngine, group=None) -> Callable:
    """In-place sum over the ranks on the engine's stream (NCCL)."""
    import torch
    import torch.distributed as dist

    def reduce(buf):
        if dist.is_initialized() and dist.get_world_size(group) > 1:
            with torch.cuda.stream(engine.stream):
                dist.all_reduce(buf, group=group)
    return reduce


def host_reduce(engine: DeviceEngine, group=None) -> Callable:
    """In-place sum over the ranks through host memory, for process groups
    whose backend reduces host tensors only (gloo): the buffer is copied to
    the host once the engine's stream has produced it, summed, and copied
    back on the engine's stream."""
    import torch
    import torch.distributed as dist

    def reduce(buf):
        if dist.is_initialized() and dist.get_world_size(group) > 1:
            with torch.cuda.stream(engine.stream):
                h = buf.cpu()  # waits for the engine's stream
            dist.all_reduce(h, group=group)
            with torch.cuda.stream(engine.stream):
                buf.copy_(h)
    return reduce
