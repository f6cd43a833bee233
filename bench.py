"""Benchmark of the B200 FD engine -- one JSON line on stdout (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload lsrtm_large|lsrtm_1200x400]

Workload ``lsrtm_large`` (default): least-squares RTM by CG (CGLS) on the
largest survey -- 4000 x 1000 cells at 5 m, pml 40, nt 8000 + 120 delay steps,
dt 0.5 ms, 25 Hz Ricker, 256 shots with apertures of 1000-4000 columns drawn
from a seed, layered model with velocity anomalies.  Velocities are capped at
3000 m/s: at this survey's 5500 m/s (Courant number 0.55) the reference's
scheme -- its absorbing boundary, which this library reproduces bit for bit --
grows without bound over 8120 steps from a Courant number of about 0.33 up.
One GPU runs a sample of 8 of the 256 shots (shots 0, 32, ..., 224; under
torchrun rank r takes shots r, 32 + r, ...: weak scaling, no collective on
the data path), with the solver as the full survey needs it on a GPU: FP16
source-term snapshots every 4 steps with one power-of-two scale per tile,
source-field checkpoints every 256 steps, FP64 CG scalars.  One step = one CG
iteration over the sample: Born modeling of its 8 shots (two fields per step),
their exact adjoint (reverse pass plus the recomputed source field of each
checkpoint segment) and the FP64 vector algebra.  Metric: padded grid
cell-updates per second (Gcell/s), whole job; ``ms_per_step`` is the
iteration time.

* ``value``: device-resident solver state, CUDA-event timed iterations.
* ``e2e``: the public LSRTM API with host buffers, every step: background and
  wavelet upload, the observed data of every shot from pinned memory, reset
  (checkpoint pass + first adjoint), one iteration, model download.
* ``plain_fp32``: the same Born + adjoint work on the plain path -- one shot
  per plan and launch sequence, FP32 source snapshots at every step (with the
  same checkpoints: kept whole they take ~40 GB per wide shot), the source
  pass made per shot -- timed on every shot of the sample: ``iter_ms`` with
  the plans built and run as a per-shot path does in every CG iteration,
  ``iter_ms_warm`` the same plans run again (device work only); the config
  carries both ratios.
  ``mixed_regrouped``: the batched mixed solver rebuilding its plans in every
  operator application (shot-group mode, as on one GPU for all 256 shots),
  which also redoes the checkpoint pass: it separates batching and mixed
  storage from the reuse of the source field across iterations.
* ``image_error``: the first CG gradient image L^T d of one shot (shot 64)
  from the mixed-storage and the plain FP32 adjoints, against the FP64 image
  of the same shot and data (the restatement's double build, computed offline
  by tests/golden/make_large_fp64.py; compared on its stored subsample), and
  mixed against plain over all 8 shots.
* ``roofline``: the kernel with the largest share of the iteration (mean
  CUDA-event duration of the kernel alone x launches per iteration),
  algorithmic bytes per launch (16 B per field cell-update: read prev, cur,
  velocity, write next) over that duration, against the measured HBM copy
  bandwidth; rows for the interior and pad kernels of the Born step, the
  reverse step and the recomputed source-field step, and each step as run.
* ``cpu_baseline``: the reference's own ``forward`` (Born) and ``adjoint``
  (RTM) (src/util/fd.cpp:81-177, :592-719, compiled from its sources into
  oracle/_ref) on the sample's narrowest shot with the recorded samples cut
  to 24 (the 120 delay steps all run), all host threads, as cell-updates per
  second of the same work.

Workload ``lsrtm_1200x400``: one CG iteration of the 32-shot 1200 x 400 survey
(10 m, nt 5000 + 94, dt 0.8 ms, 20 Hz, FP16 snapshots every 4 steps kept
whole, no checkpoints).
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
SNAP_EVERY = 4
CK_EVERY = 256      # lsrtm_large: source-field checkpoint interval
SAMPLE = 8          # lsrtm_large: shots per GPU
STRIDE = 32         # lsrtm_large: shot index stride of a GPU's sample
FP64_SHOT = 64      # lsrtm_large: the shot with an FP64 image fixture


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


def load_synth():
    """seis_b200/synth.py loaded as a module of its own (numpy and scipy only),
    so that the reference arm builds the same inputs without importing this
    package or loading its CUDA library."""
    import importlib.util
    path = os.path.join(ROOT, "seis_b200", "synth.py")
    spec = importlib.util.spec_from_file_location("seis_bench_synth", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(name: str, rank: int, world: int, shots: int = None, nt: int = None):
    """(whole survey, this rank's shot indices, solver options); `shots` (per
    GPU) and `nt` (recorded samples) default to the workload's own."""
    synth = load_synth()
    if name == "lsrtm_large":
        k = min(shots or SAMPLE, SAMPLE)
        full = synth.large_sweep(vmax=3000.0, nt=nt or 8000)
        mine = [j * STRIDE + rank for j in range(k)]
        return full, mine, {"checkpoint_every": CK_EVERY}
    if name == "lsrtm_1200x400":
        k = shots or 32
        full = synth.lsrtm(nshots=k * world, nt=nt or 5000)
        mine = list(range(k * rank, k * rank + k))
        return full, mine, {"checkpoint_every": 0}
    raise SystemExit(f"unknown workload {name}")


def config_of(name: str, full, sv, world: int) -> dict:
    """The workload's `config`, the same for both arms."""
    s0 = sv.shots[0]
    c = {"workload": name, "shots_per_gpu": len(sv.shots), "shots_total_survey": len(full.shots),
         "shots_timed_total": len(sv.shots) * world, "apertures_rank0": [s.nx for s in sv.shots],
         "grid": f"{full.nx}x{full.nz} at {full.dx:g} m, pml {s0.pml}",
         "nt": s0.nt, "ndel": s0.ndel, "dt_s": s0.dt, "ricker_hz": full.fr,
         "snapshots": f"FP16 every {SNAP_EVERY} steps, per-tile power-of-two scale",
         "step": "one CG iteration over the GPU's shots: Born of every shot, its exact "
                 "adjoint, FP64 CG algebra",
         "exchange": "per CG iteration: NCCL all-reduce of the image and 2 FP64 sums"
                     if world > 1 else "none"}
    if name == "lsrtm_large":
        c.update({"velocity_cap_m_s": 3000.0, "checkpoint_every": CK_EVERY,
                  "shot_indices_rank0": [k * STRIDE for k in range(len(sv.shots))],
                  "sample": f"{len(sv.shots)} of the survey's {len(full.shots)} shots per GPU "
                            f"(every {STRIDE}th)"})
    return c


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(sv, steps_cap: int):
    """The reference's `forward` (Born) and `adjoint` (RTM), compiled from its
    own sources, on the sample's narrowest shot with the recorded time samples
    cut to `steps_cap` (the delay steps all run); rate = the cell-updates of
    one CG iteration of that shot and step count (3 NT + 1 per padded cell:
    Born two fields, adjoint one) over the reference's Born + adjoint time,
    i.e. the reference's speed on the same job."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dataclasses

    import oracle as O
    k = min(range(len(sv.shots)), key=lambda i: sv.shots[i].nx)
    s0 = sv.shots[k]
    s = dataclasses.replace(s0, nt=steps_cap)
    kind = "reference" if O.ref_available() else "port"
    impl = "ref" if kind == "reference" else "oracle"
    wav = sv.wavelet(lambda dt, fr, d, n: O.ricker(dt, fr, d, n, impl=impl))[:s.NT]
    vel, dv = sv.sub(sv.vel0, k), sv.sub(sv.dv, k)
    cores = len(os.sched_getaffinity(0))
    if kind == "reference":
        O.ref_set_threads(cores)
    else:
        cores = 1
    t = time.perf_counter()
    rec = O.born(s, wav, vel, dv, impl=impl)
    t_born = time.perf_counter() - t
    t = time.perf_counter()
    O.rtm(s, wav, vel, rec, impl=impl)
    t_adj = time.perf_counter() - t
    dt = t_born + t_adj
    cells = (s.nx + 2 * s.pml) * (s.nz + 2 * s.pml) * (3 * s.NT + 1)
    return {"value": cells / dt / 1e9, "unit": "Gcell/s", "cores": cores, "kind": kind,
            "cpu": cpu_model(),
            "sample": f"forward (Born) {t_born:.2f} s + adjoint (RTM) {t_adj:.2f} s of one shot "
                      f"({s.nx}x{s.nz}, pml {s.pml}), {s.NT} of {s0.NT} steps; the reference has "
                      f"no CG, so one iteration = these two calls per shot"}


def synth_data_note(name: str) -> str:
    if name == "lsrtm_large":
        return ("synthetic (seeded 4000x1000 layered model with Gaussian anomalies, capped at "
                "3000 m/s; observed data = Born modeling of the true perturbation)")
    return ("synthetic (seeded layered + faulted 1200x400 model; observed data = Born modeling "
            "of the true perturbation)")


def run_reference(args, rank, world):
    """The reference's CPU path on this workload (bounded sample per step)."""
    if rank != 0:
        return
    full, mine, _ = workload(args.workload, rank, world, args.shots, args.nt)
    sv = full.subset(mine)
    cap = 24 if args.workload == "lsrtm_large" else 150
    vals, last = [], None
    for i in range(args.warmup + args.steps):
        last = cpu_baseline(sv, steps_cap=cap)
        if i >= args.warmup:
            vals.append(last["value"])
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": "Gcell-updates/s", "value": v, "unit": "Gcell/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": synth_data_note(args.workload),
            "config": config_of(args.workload, full, sv, world),
            "cpu_baseline": {"value": v, "unit": "Gcell/s", "cores": last["cores"],
                             "kind": last["kind"], "cpu": last["cpu"], "sample": last["sample"]},
            "e2e": {"value": v, "unit": "Gcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def observed_data(ctx, sv):
    """Synthetic observed data: Born gathers of the true perturbation over the
    background, exact-rounding kernels (equal to the reference's own Born)."""
    from seis_b200._lib import IN_DV, IN_VEL, IN_WAVELET, OP_BORN, OUT_GATHER, Plan
    wav = sv.wavelet()
    out = []
    for i in range(len(sv.shots)):  # one at a time: the widest gathers are 130 MB
        with Plan(ctx, OP_BORN, [sv.shots[i]]) as p:
            p.set(0, IN_VEL, sv.sub(sv.vel0, i))
            p.set(0, IN_DV, sv.sub(sv.dv, i))
            p.set(0, IN_WAVELET, wav)
            p.run()
            out.append(p.get(0, OUT_GATHER))
    return out


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per cell of one
# launch of each step kernel, from the ncu captures summarised in profiles/
# (16 shots of the 1200 x 400 survey; Born kernels at 32 x 32 tiles, adjoint
# kernels at 64 x 32); a launch's traffic is this times the cells it
# updates (the captures' halo overhead is that of their tile shapes).
NCU_TRAFFIC_PER_CELL = {
    "born_interior": 215.0e6 / (6336 * 1024),
    "born_pad": 141.0e6 / (3264 * 1024),
    "adjoint_interior": 97.4e6 / (103809024 / 16),
    "adjoint_pad": 127.2e6 / (1632 * 2048),
}


def kernel_roofline(ctx, sv, iter_ms, launches_per_iter):
    """Per-kernel CUDA-event durations of the step kernels of one iteration --
    the Born step, the adjoint's reverse step and the source-field step it
    recomputes per checkpoint segment -- on separate plans over the same
    shots: every kernel timed alone (interior tiles, then pad tiles), and the
    step as a run launches it (both kernels, concurrently).  Returns the row
    of the kernel with the largest share of the iteration (alone-time x
    launches), every row, and the autotuner's step times per tile shape."""
    from seis_b200._lib import (IN_DV, IN_VEL, IN_WAVELET, OP_BORN, OP_BORN_ADJOINT, OP_MODELING,
                                TILE_SHAPES, Plan)
    wav = sv.wavelet()
    rows, tuning = [], {}
    for op, name in ((OP_BORN, "born"), (OP_BORN_ADJOINT, "adjoint"), (OP_MODELING, "source")):
        n = launches_per_iter.get(name, 0)
        if not n:
            continue
        with Plan(ctx, op, sv.shots) as p:
            if op != OP_BORN_ADJOINT:
                p.set_exact(False)  # the solver's forward operators run the fast build
            for i in range(len(sv.shots)):
                p.set(i, IN_VEL, sv.sub(sv.vel0, i))
                p.set(i, IN_WAVELET, wav)
                if op == OP_BORN:
                    p.set(i, IN_DV, sv.sub(sv.dv, i))
            if op != OP_MODELING:
                # the autotuner's step time of every tile shape on these shots
                # (the solver's plans of the same signature use the same choice)
                best, per_shape = p.autotune(steps=10, force=True)
                tuning[name] = {"chosen": "%dx%d" % TILE_SHAPES[best],
                                "step_ms": {"%dx%d" % TILE_SHAPES[k]: v
                                            for k, v in enumerate(per_shape)}}
            p.time_kernels(10)
            ms, by = p.time_kernels(100)
        per_cell = 32.0 if op == OP_BORN else 16.0
        for k, kname in ((0, "interior"), (1, "pad")):
            kern = f"{name}_{kname}"
            tr = NCU_TRAFFIC_PER_CELL.get(kern)
            rows.append({"kernel": kern, "ms": ms[k], "bytes": by[k], "launches_per_iter": n,
                         "share": ms[k] * n / iter_ms, "GB_s": by[k] / (ms[k] * 1e6),
                         "traffic": tr * by[k] / per_cell if tr else None, "timed": "alone"})
        rows.append({"kernel": f"{name}_step", "ms": ms[2], "bytes": by[0] + by[1],
                     "launches_per_iter": n, "share": ms[2] * n / iter_ms,
                     "GB_s": (by[0] + by[1]) / (ms[2] * 1e6), "timed": "as run"})
    kern = [r for r in rows if not r["kernel"].endswith("_step")]
    top = max(kern, key=lambda r: r["ms"] * r["launches_per_iter"])
    return top, rows, tuning


def adjoint_images(ctx, sv, dobs, every, dtype, ck):
    """Per-shot exact-adjoint images L_s^T d_s (one batched plan)."""
    from seis_b200._lib import IN_GATHER, IN_VEL, IN_WAVELET, OP_BORN_ADJOINT, OUT_IMAGE, Plan
    wav = sv.wavelet()
    with Plan(ctx, OP_BORN_ADJOINT, sv.shots) as p:
        p.set_snapshots(every, dtype)
        if ck:
            p.set_checkpoints(ck)
        for i in range(len(sv.shots)):
            p.set(i, IN_VEL, sv.sub(sv.vel0, i))
            p.set(i, IN_WAVELET, wav)
            p.set(i, IN_GATHER, dobs[i])
        p.run()
        return [p.get(i, OUT_IMAGE) for i in range(len(sv.shots))]


def plain_fp32(ctx, sv, dobs, ck):
    """The Born + adjoint work of one CG iteration on the plain path, every
    shot of the sample: per shot one single-shot Born plan (FP32, fast build)
    and one single-shot adjoint plan with FP32 snapshots at every step (and
    the solver's checkpoints), source pass per shot.  Timed twice per shot:
    cold -- the plans built, their inputs uploaded and run once, as a
    per-shot path does in every CG iteration (graph capture included); warm
    -- the same plans run again (the velocity set again, so that the source
    field is recomputed): the device work alone.
    Returns (cold seconds, warm seconds, per-shot images of the adjoint)."""
    import torch
    from seis_b200._lib import (IN_DV, IN_GATHER, IN_VEL, IN_WAVELET, OP_BORN, OP_BORN_ADJOINT,
                                OUT_IMAGE, SNAP_F32, Plan)
    wav = sv.wavelet()
    p0 = np.ones((sv.nx, sv.nz), np.float32)
    imgs = []
    cold = warm = 0.0
    for i, s in enumerate(sv.shots):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with Plan(ctx, OP_BORN, [s]) as pb, Plan(ctx, OP_BORN_ADJOINT, [s]) as pa:
            pb.set_exact(False)
            pb.set(0, IN_VEL, sv.sub(sv.vel0, i))
            pb.set(0, IN_WAVELET, wav)
            pb.set(0, IN_DV, sv.sub(p0, i))
            pb.run()
            pa.set_snapshots(1, SNAP_F32)
            if ck:
                pa.set_checkpoints(ck)
            pa.set(0, IN_VEL, sv.sub(sv.vel0, i))
            pa.set(0, IN_WAVELET, wav)
            pa.set(0, IN_GATHER, dobs[i])
            pa.run()
            pa.sync()
            cold += time.perf_counter() - t0
            pa.set(0, IN_VEL, sv.sub(sv.vel0, i))  # the source pass runs again
            pa.sync()
            t0 = time.perf_counter()
            pb.run()
            pa.run()
            pa.sync()
            warm += time.perf_counter() - t0
            imgs.append(pa.get(0, OUT_IMAGE))
    return cold, warm, imgs


def image_errors(mine, img_mixed, img_plain):
    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out = {"mixed_vs_plain_all_shots": rel(np.concatenate([x.ravel() for x in img_mixed]),
                                            np.concatenate([x.ravel() for x in img_plain]))}
    path = os.path.join(ROOT, "tests", "golden", "large_fp64.npz")
    if FP64_SHOT in mine and os.path.exists(path):
        g = np.load(path)
        k = mine.index(FP64_SHOT)
        st = int(g["step"])
        ref = g["img_sub"].astype(np.float64)
        out.update({
            "fp64_shot": FP64_SHOT,
            "fp64_reference": "exact Born adjoint in FP64 (the restatement's double build) of the "
                              "same shot and data, computed offline (tests/golden/"
                              f"make_large_fp64.py); compared on every {st}th column and row",
            "mixed_vs_fp64": rel(img_mixed[k][::st, ::st], ref),
            "plain_fp32_vs_fp64": rel(img_plain[k][::st, ::st], ref)})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="lsrtm_large", choices=["lsrtm_large", "lsrtm_1200x400"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--shots", type=int, default=None,
                    help="shots per GPU (default: the workload's, 8 of lsrtm_large, 32 of "
                         "lsrtm_1200x400)")
    ap.add_argument("--nt", type=int, default=None,
                    help="recorded time samples (default: the workload's)")
    args = ap.parse_args()
    rank, world, local = dist_init()
    if args.impl == "reference":
        run_reference(args, rank, world)
        barrier(world)
        return

    import torch
    from seis_b200 import Context
    from seis_b200._lib import SNAP_F16, Lsrtm

    torch.cuda.set_device(local)
    from seis_b200.shards import DeviceEngine, ShardedCGLS, nccl_reduce
    full, mine, opts = workload(args.workload, rank, world, args.shots, args.nt)
    sv = full.subset(mine)
    shots = sv.shots
    ck = opts["checkpoint_every"]
    ctx = Context(local)
    wav = sv.wavelet()
    dobs = observed_data(ctx, sv)
    ls = Lsrtm(ctx, sv.nx, sv.nz, shots, sv.x0, snap_every=SNAP_EVERY, snap_dtype=SNAP_F16,
               checkpoint_every=ck)
    ls.set_background(sv.vel0, wav)
    for i, d in enumerate(dobs):
        ls.set_data(i, d)
    eng = DeviceEngine(ls)
    cg = ShardedCGLS(eng, nccl_reduce(eng))
    rr0 = cg.reset()
    cells = ls.cell_updates

    # ---- device-resident: CG iterations timed with CUDA events on the
    # library's stream
    stream = eng.stream
    rr_warm = cg.iterate(args.warmup) if args.warmup > 0 else []
    launches0 = ctx.launches
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rr = []
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        # the timed iterations as one NVTX range ("bench_timed"), for a
        # profiler's launch list of exactly this region
        torch.cuda.nvtx.range_push("bench_timed")
        start.record(stream)
        for _ in range(args.steps):
            rr.extend(cg.iterate(1))
        stop.record(stream)
        stop.synchronize()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
    clocks = clk.summary()
    launches = ctx.launches - launches0
    ms_per_step = start.elapsed_time(stop) / args.steps
    ms_per_step = max_over_ranks(ms_per_step, world)
    value = cells * world / (ms_per_step / 1e3) / 1e9

    # ---- end to end through the public LSRTM API with pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    h_v0, h_wav = pin(sv.vel0), pin(wav)
    h_d = [pin(d) for d in dobs]
    h_m = torch.empty((sv.nx, sv.nz), dtype=torch.float32).pin_memory()
    h_rr = torch.empty(2, dtype=torch.float64)
    L = ctx.L

    def e2e_step():
        ctx.check(L.seis_fd_lsrtm_set_background(ls.h, h_v0.data_ptr(), h_wav.data_ptr()))
        for i in range(len(shots)):
            ctx.check(L.seis_fd_lsrtm_set_data(ls.h, i, h_d[i].data_ptr()))
        h_rr[0] = cg.reset()
        h_rr[1] = cg.iterate(1)[0]
        ctx.check(L.seis_fd_lsrtm_model(ls.h, h_m.data_ptr()))

    e2e_steps = max(1, args.steps // 4)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, world)
    # reset = checkpoint (or snapshot) pass + one adjoint application (with
    # checkpoints: reverse pass + recomputed source field)
    reset_cells = sum((s.nx + 2 * s.pml) * (s.nz + 2 * s.pml) *
                      (s.NT + (s.NT + 1) + (s.NT if ck else 0)) for s in shots)
    e2e_cells = (cells + reset_cells) * world
    h2d = sv.vel0.nbytes + wav.nbytes + sum(d.nbytes for d in dobs)
    d2h = h_m.numel() * 4 + 16
    dev_bytes = ls.device_bytes
    ls.close()

    # ---- the same iteration with the plans rebuilt in every application
    regroup = None
    if world == 1 and not args.no_plain and args.workload == "lsrtm_large":
        with Lsrtm(ctx, sv.nx, sv.nz, shots, sv.x0, snap_every=SNAP_EVERY, snap_dtype=SNAP_F16,
                   checkpoint_every=ck, group_shots=len(shots)) as lg:
            lg.set_background(sv.vel0, wav)
            for i, d in enumerate(dobs):
                lg.set_data(i, d)
            lg.reset()
            lg.iterate(1)
            torch.cuda.synchronize()
            t = time.perf_counter()
            lg.iterate(1)
            torch.cuda.synchronize()
            regroup = {"iter_ms": (time.perf_counter() - t) * 1e3,
                       "how": "the batched mixed solver in shot-group mode: the plans of the "
                              "group built in every operator application, checkpoint pass redone"}

    # ---- plain FP32 path and image errors
    plain = errors = None
    if world == 1 and not args.no_plain:
        t_cold, t_warm, img_plain = plain_fp32(ctx, sv, dobs, ck)
        img_mixed = adjoint_images(ctx, sv, dobs, SNAP_EVERY, SNAP_F16, ck)
        plain = {"iter_ms": t_cold * 1e3, "iter_ms_warm": t_warm * 1e3, "shots": len(shots),
                 "how": "one shot per plan and graph; Born run, then the exact adjoint with FP32 "
                        "snapshots at every step" + (f" (checkpoints every {ck} steps)" if ck else "")
                        + ", source pass per shot; every shot of the sample timed. iter_ms: "
                          "plans built, uploaded and run (as in every CG iteration of a per-shot "
                          "path); iter_ms_warm: the same plans run again (device work only)"}
        errors = image_errors(mine, img_mixed, img_plain)

    # ---- roofline of the kernel with the largest share
    # per iteration: the Born steps, the reverse steps, and with checkpoints
    # the source-field steps recomputed segment by segment
    per_iter_launches = {"born": shots[0].NT, "adjoint": shots[0].NT + 1,
                         "source": shots[0].NT if ck else 0}
    top, rows, tuning = kernel_roofline(ctx, sv, ms_per_step, per_iter_launches)
    hbm, src = peaks()
    ach = top["bytes"] / (top["ms"] * 1e-3) / 1e9
    line = {
        "metric": "Gcell-updates/s", "value": value, "unit": "Gcell/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": synth_data_note(args.workload),
        "config": config_of(args.workload, full, sv, world),
        "e2e": {"value": e2e_cells / (e2e_ms / 1e3) / 1e9, "unit": "Gcell/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "cell_updates_per_step": e2e_cells},
        "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                     "frac": ach / hbm, "traffic": top.get("traffic"),
                     "traffic_unit": "bytes per launch (ncu dram read + write, scaled by cells)",
                     "kernel": top["kernel"], "peak_source": src, "kernel_ms": top["ms"],
                     "share": top["share"], "kernels": rows},
        "tile_shapes": tuning,
        "gpu_launches": launches,
        "clocks": clocks,
    }
    cfg = line["config"]
    cfg.update({"cell_updates_per_step": cells, "lsrtm_iter_ms": ms_per_step,
                "device_bytes": dev_bytes,
                "l2": "inputs larger than L2: fields, checkpoints, snapshots and data of the "
                      f"shots ({dev_bytes / 2**30:.1f} GiB resident)",
                "residual": {"rr0": rr0, "after_warmup": list(map(float, rr_warm)),
                             "timed": rr}})
    if plain:
        line["plain_fp32"] = plain
        cfg["speedup_vs_plain_fp32"] = plain["iter_ms"] / ms_per_step
        cfg["speedup_vs_plain_fp32_warm"] = plain["iter_ms_warm"] / ms_per_step
    if regroup:
        line["mixed_regrouped"] = regroup
        if plain:
            cfg["speedup_regrouped_vs_plain_fp32"] = plain["iter_ms"] / regroup["iter_ms"]
    if errors:
        line["image_error"] = errors
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sv, 24 if args.workload == "lsrtm_large" else 150)
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
