"""Benchmark of the B200 FD engine -- one JSON line on stdout (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload born_lsrtm]

Workload ``born_lsrtm`` (default): linearised Born modeling of all 32 shots of
the 1200x400 LSRTM survey (10 m grid, pml 40, nt 5000 + 94 delay steps,
dt 0.8 ms, 20 Hz Ricker, full-aperture receivers at gz=1), i.e. the forward
half of one LSRTM CG iteration.  One step = one batched Born run of the 32
shots (two fields advanced per time step).  Metric: padded grid cell-updates
per second (Gcell/s), whole job.

* ``value``: device-resident inputs, CUDA-event timed graph replays.
* ``e2e``: the same through the public plan API with host buffers: every step
  uploads velocity, perturbation and wavelet of every shot from pinned memory
  and downloads every gather.
* ``roofline``: the interior-tile kernel (dominant), algorithmic bytes per
  launch (16 B per field-update: read prev, cur, vel; write next -- the Born
  kernel also reads dv, counted inside 16 B x 2 fields) over its mean
  CUDA-event duration, against the measured HBM copy bandwidth.
* ``cpu_baseline``: the reference's own ``forward`` (src/util/fd.cpp:81-177,
  compiled from its sources into oracle/_ref) on one shot of the workload with
  the time loop cut to a bounded number of steps, all host threads.

Under torchrun (N > 1) every rank runs its own 32-shot survey (weak scaling);
there is no data-path collective in this workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 2 ** 20


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"seis_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload(name: str, rank: int):
    from seis_b200 import synth
    if name == "born_lsrtm":
        return synth.lsrtm()
    raise SystemExit(f"unknown workload {name}")


def cpu_baseline(sv, steps_cap: int = 300):
    """Reference `forward` (compiled from its own sources) on shot 0 of the
    survey, time loop cut to `steps_cap` recorded samples."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    s0 = sv.shots[0]
    from seis_b200 import Shot
    s = Shot(nx=s0.nx, nz=s0.nz, pml=s0.pml, nt=steps_cap, ndel=s0.ndel, sx=s0.sx, sz=s0.sz,
             dt=s0.dt, dx=s0.dx, dz=s0.dz, gz=s0.gz)
    wav = sv.wavelet()[:s.NT]
    vel, dv = sv.sub(sv.vel0, 0), sv.sub(sv.dv, 0)
    kind = "reference" if O.ref_available() else "port"
    cores = len(os.sched_getaffinity(0))
    if kind == "reference":
        O.ref_set_threads(cores)
    t = time.perf_counter()
    if kind == "reference":
        O.born(s, wav, vel, dv, impl="ref")
    else:
        cores = 1
        O.born(s, wav, vel, dv)
    dt = time.perf_counter() - t
    cells = 2 * (s.nx + 2 * s.pml) * (s.nz + 2 * s.pml) * s.NT
    return {"value": cells / dt / 1e9, "unit": "Gcell/s", "cores": cores, "kind": kind,
            "sample": f"Born of shot 0 ({s.nx}x{s.nz}, pml {s.pml}), {s.NT} of {s0.NT} steps, "
                      f"{dt:.2f} s"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    sv = workload(args.workload, rank)
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(sv, steps_cap=120 if i < args.warmup else 200)
        if i >= args.warmup:
            vals.append(r["value"])
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": "Gcell-updates/s", "value": v, "unit": "Gcell/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": args.workload},
            "cpu_baseline": {"value": v, "unit": "Gcell/s", "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
            "e2e": {"value": v, "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="born_lsrtm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank, world, local = dist_init()
    if args.impl == "reference":
        run_reference(args, rank, world)
        barrier(world)
        return

    import torch
    from seis_b200 import Context
    from seis_b200._lib import IN_DV, IN_VEL, IN_WAVELET, OP_BORN, OUT_GATHER, Plan, ptr

    torch.cuda.set_device(local)
    sv = workload(args.workload, rank)
    shots = sv.shots
    ctx = Context(local)
    plan = Plan(ctx, OP_BORN, shots)
    wav = sv.wavelet()
    vels = [sv.sub(sv.vel0, i) for i in range(len(shots))]
    dvs = [sv.sub(sv.dv, i) for i in range(len(shots))]
    for i in range(len(shots)):
        plan.set(i, IN_VEL, vels[i])
        plan.set(i, IN_DV, dvs[i])
        plan.set(i, IN_WAVELET, wav)
    cells = plan.cell_updates

    # ---- device-resident: graph replays timed with CUDA events on the
    # library's stream
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=torch.device("cuda", local))
    for _ in range(args.warmup):
        plan.run()
    plan.sync()
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            plan.run()
        stop.record(stream)
        stop.synchronize()
        torch.cuda.synchronize()
    clocks = clk.summary()
    ms_per_step = start.elapsed_time(stop) / args.steps
    ms_per_step = max_over_ranks(ms_per_step, world)
    value = cells * world / (ms_per_step / 1e3) / 1e9

    # ---- end to end through the plan API with pinned host buffers
    pin = lambda a: torch.from_numpy(a).pin_memory()
    h_vel = [pin(v) for v in vels]
    h_dv = [pin(d) for d in dvs]
    h_wav = pin(wav)
    h_rec = [torch.empty((s.nx, s.nt), dtype=torch.float32).pin_memory() for s in shots]
    L = ctx.L

    def e2e_step():
        for i in range(len(shots)):
            ctx.check(L.seis_fd_plan_set(plan.h, i, IN_VEL, h_vel[i].data_ptr()))
            ctx.check(L.seis_fd_plan_set(plan.h, i, IN_DV, h_dv[i].data_ptr()))
            ctx.check(L.seis_fd_plan_set(plan.h, i, IN_WAVELET, h_wav.data_ptr()))
        plan.run()
        for i in range(len(shots)):
            ctx.check(L.seis_fd_plan_get(plan.h, i, OUT_GATHER, h_rec[i].data_ptr()))

    e2e_step()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        e2e_step()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / max(1, args.steps // 2)
    e2e_ms = max_over_ranks(e2e_ms, world)
    h2d = sum(v.nbytes + d.nbytes + wav.nbytes for v, d in zip(vels, dvs))
    d2h = sum(s.nx * s.nt * 4 for s in shots)

    # ---- roofline of the dominant kernel
    ms, by = plan.time_kernels(200)
    hbm, src = peaks()
    ach = by[0] / (ms[0] * 1e-3) / 1e9
    line = {
        "metric": "Gcell-updates/s", "value": value, "unit": "Gcell/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": args.workload, "shots_per_gpu": len(shots), "grid": "1200x400 pml 40",
                   "nt": shots[0].nt, "ndel": shots[0].ndel, "fields": 2,
                   "cell_updates_per_step": cells, "l2": "inputs larger than L2 "
                   f"({(sum(v.nbytes for v in vels) * 8) / 2**20:.0f} MiB working set)"},
        "e2e": {"value": cells * world / (e2e_ms / 1e3) / 1e9, "unit": "Gcell/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                     "frac": ach / hbm, "traffic": None, "kernel": "interior_kernel<BORN>",
                     "peak_source": src, "interior_ms": ms[0], "boundary_ms": ms[1],
                     "step_ms": ms[2]},
        "gpu_launches": plan.launches_per_run * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sv)
    plan.close()
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
