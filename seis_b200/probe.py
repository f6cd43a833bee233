"""Measurement programs.

    python -m seis_b200.probe {born|modeling|adjoint} [--steps K] [--nt NT] [--exact]

Per-kernel timing of one operator's step kernels on the LSRTM survey (32
shots, 1200 x 400 model): the program the profiles under profiles/ are
captured from.  Prints the interior-tile, pad-path and whole-step milliseconds
(CUDA events, kernels concurrent as in a run) and the algorithmic bytes of
each.

    python -m seis_b200.probe large [--shots N]

A sample of the large survey (4000 x 1000 cells at 5 m, nt 8000, apertures
1000-4000 columns; its BF16 snapshots alone take ~16 GB per full-aperture
shot), velocities capped at 3000 m/s (Courant number 0.30: over 8000 steps
with a 40-cell pad the reference's own scheme grows without bound from about
0.33 up, and the survey reaches 0.55): one LSRTM CG
iteration of N shots (default 4) batched with BF16 snapshots every 4 steps,
kept whole and with source-field checkpoints every 256 steps, against the
plain path -- one shot per plan, FP32 snapshots at every step (checkpointed
too: they would need ~130 GB per shot), source pass made per shot -- and the
adjoint images of the two against each other.

    python -m seis_b200.probe snapshots [--nt NT]

Snapshot storage on the batched survey (64 shots of uneven aperture, 300-737
columns, on the 737 x 240 layered model with anomalies): the exact adjoint of
every shot, residuals = Born data of the true perturbation, in one plan per
storage choice -- FP32 at every step (with source-field checkpoints: keeping
them all would take ~130 GB), FP32 / BF16 / FP16 every 4 steps, BF16 every 4
steps with checkpoints.  Prints per choice the image error (relative L2 over
all shots) against FP32 at every step, the time of one run (graph replay,
snapshots already made, or recomputed per segment with checkpoints), its
cell-update rate and the plan's device memory.
"""
from __future__ import annotations

import argparse
import json


def snapshots(nt: int) -> dict:
    import time

    import numpy as np

    from . import Context, synth
    from ._lib import (IN_DV, IN_GATHER, IN_VEL, IN_WAVELET, OP_BORN, OP_BORN_ADJOINT, OUT_GATHER,
                       OUT_IMAGE, SNAP_BF16, SNAP_F16, SNAP_F32, Plan)
    sv = synth.batched_rtm(nt=nt)
    wav = sv.wavelet()
    n = len(sv.shots)
    out = {"survey": f"{n} shots, apertures {min(s.nx for s in sv.shots)}-"
                     f"{max(s.nx for s in sv.shots)} columns of {sv.nx} x {sv.nz}, nt {nt}"}
    with Context(0) as ctx:
        with Plan(ctx, OP_BORN, sv.shots) as p:
            p.set_exact(False)
            for i in range(n):
                p.set(i, IN_VEL, sv.sub(sv.vel0, i))
                p.set(i, IN_DV, sv.sub(sv.dv, i))
                p.set(i, IN_WAVELET, wav)
            p.run()
            data = [p.get(i, OUT_GATHER) for i in range(n)]
        choices = [("f32_every1_ck64", 1, SNAP_F32, 64), ("f32_every4", 4, SNAP_F32, 0),
                   ("bf16_every4", 4, SNAP_BF16, 0), ("f16_every4", 4, SNAP_F16, 0),
                   ("bf16_every4_ck64", 4, SNAP_BF16, 64)]
        ref = None
        for name, every, dtype, ck in choices:
            with Plan(ctx, OP_BORN_ADJOINT, sv.shots) as p:
                p.set_snapshots(every, dtype)
                if ck:
                    p.set_checkpoints(ck)
                for i in range(n):
                    p.set(i, IN_VEL, sv.sub(sv.vel0, i))
                    p.set(i, IN_WAVELET, wav)
                    p.set(i, IN_GATHER, data[i])
                p.run()  # source pass (snapshots or checkpoints) and graph capture
                p.sync()
                t = time.perf_counter()
                p.run()
                p.sync()
                sec = time.perf_counter() - t
                img = np.concatenate([p.get(i, OUT_IMAGE).ravel() for i in range(n)]).astype(
                    np.float64)
                cells = p.cell_updates
                if ck == 0:  # the source pass is not part of a replayed run
                    cells -= sum(sv.cell_updates_of(i) for i in range(n))
                row = {"run_s": sec, "Gcell_s": cells / sec / 1e9,
                       "device_GB": p.device_bytes / 1e9}
            if ref is None:
                ref = img
            row["image_rel_l2_vs_f32_every1"] = float(np.linalg.norm(img - ref) / np.linalg.norm(ref))
            out[name] = row
    return out


def large(nshots: int) -> dict:
    import time

    import numpy as np

    from . import Context, synth
    from ._lib import (IN_DV, IN_GATHER, IN_VEL, IN_WAVELET, OP_BORN, OP_BORN_ADJOINT, OUT_GATHER,
                       OUT_IMAGE, SNAP_BF16, SNAP_F32, Lsrtm, Plan)
    sv = synth.large_sweep(vmax=3000.0).subset(range(nshots))
    wav = sv.wavelet()
    n, CK = len(sv.shots), 256
    out = {"sample": f"{n} shots of the large survey, apertures "
                     f"{', '.join(str(s.nx) for s in sv.shots)} columns of {sv.nx} x {sv.nz}, "
                     f"NT {sv.shots[0].NT}"}
    with Context(0) as ctx:
        with Plan(ctx, OP_BORN, sv.shots) as p:
            p.set_exact(False)
            for i in range(n):
                p.set(i, IN_VEL, sv.sub(sv.vel0, i))
                p.set(i, IN_DV, sv.sub(sv.dv, i))
                p.set(i, IN_WAVELET, wav)
            p.run()
            data = [p.get(i, OUT_GATHER) for i in range(n)]
        out["data_finite"] = [bool(np.isfinite(d).all()) for d in data]
        out["data_max_abs"] = [float(np.nanmax(np.abs(d))) for d in data]
        # mixed storage, batched: one CG iteration, snapshots kept whole and
        # with checkpoints
        for name, ck in (("mixed_batched", 0), ("mixed_batched_checkpoints", CK)):
            with Lsrtm(ctx, sv.nx, sv.nz, sv.shots, sv.x0, snap_every=4, snap_dtype=SNAP_BF16,
                       checkpoint_every=ck) as ls:
                ls.set_background(sv.vel0, wav)
                for i, d in enumerate(data):
                    ls.set_data(i, d)
                t = time.perf_counter()
                rr0 = ls.reset()
                t_reset = time.perf_counter() - t
                rr1 = ls.iterate(1)
                t = time.perf_counter()
                rr2 = ls.iterate(1)
                t_iter = time.perf_counter() - t
                out[name] = {"iter_s": t_iter, "reset_s": t_reset,
                             "Gcell_s": ls.cell_updates / t_iter / 1e9,
                             "device_GB": ls.device_bytes / 1e9,
                             "residuals": [float(rr0), float(rr1[0]), float(rr2[0])]}
        # the adjoint images of both storage choices, and the plain iteration:
        # per shot one Born run and one adjoint run (source pass included)
        img_mixed, img_plain, t_plain = [], [], 0.0
        with Plan(ctx, OP_BORN_ADJOINT, sv.shots) as p:
            p.set_snapshots(4, SNAP_BF16)
            p.set_checkpoints(CK)
            for i in range(n):
                p.set(i, IN_VEL, sv.sub(sv.vel0, i))
                p.set(i, IN_WAVELET, wav)
                p.set(i, IN_GATHER, data[i])
            p.run()
            img_mixed = [p.get(i, OUT_IMAGE) for i in range(n)]
        one = np.ones((sv.nx, sv.nz), np.float32)
        for i, s in enumerate(sv.shots):
            with Plan(ctx, OP_BORN, [s]) as pb, Plan(ctx, OP_BORN_ADJOINT, [s]) as pa:
                pa.set_snapshots(1, SNAP_F32)
                pa.set_checkpoints(CK)
                pb.set_exact(False)
                t = time.perf_counter()
                pb.set(0, IN_VEL, sv.sub(sv.vel0, i))
                pb.set(0, IN_WAVELET, wav)
                pb.set(0, IN_DV, sv.sub(one, i))
                pb.run()
                pa.set(0, IN_VEL, sv.sub(sv.vel0, i))
                pa.set(0, IN_WAVELET, wav)
                pa.set(0, IN_GATHER, data[i])
                pa.run()
                pa.sync()
                t_plain += time.perf_counter() - t
                img_plain.append(pa.get(0, OUT_IMAGE))
        out["images_finite"] = {"mixed": [bool(np.isfinite(x).all()) for x in img_mixed],
                                "plain": [bool(np.isfinite(x).all()) for x in img_plain]}
        a = np.concatenate([x.ravel() for x in img_mixed]).astype(np.float64)
        b = np.concatenate([x.ravel() for x in img_plain]).astype(np.float64)
        out["plain_fp32"] = {"iter_s": t_plain}
        out["speedup_mixed_vs_plain"] = t_plain / out["mixed_batched"]["iter_s"]
        out["speedup_mixed_checkpoints_vs_plain"] = (
            t_plain / out["mixed_batched_checkpoints"]["iter_s"])
        out["image_rel_l2_bf16_every4_vs_fp32_every1"] = float(np.linalg.norm(a - b) /
                                                             np.linalg.norm(b))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m seis_b200.probe")
    ap.add_argument("op", choices=["born", "modeling", "adjoint", "snapshots", "large"])
    ap.add_argument("--shots", type=int, default=4, help="large: shots of the sample")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--nt", type=int, default=None,
                    help="time samples (default 400; snapshots: 4000)")
    ap.add_argument("--exact", action="store_true")
    a = ap.parse_args(argv)
    if a.op == "large":
        print(json.dumps(large(a.shots)))
        return 0
    if a.op == "snapshots":
        print(json.dumps(snapshots(a.nt or 4000)))
        return 0
    a.nt = a.nt or 400
    from . import Context, synth
    from ._lib import (IN_DV, IN_VEL, IN_WAVELET, OP_BORN, OP_BORN_ADJOINT, OP_MODELING, Plan)
    op = {"born": OP_BORN, "modeling": OP_MODELING, "adjoint": OP_BORN_ADJOINT}[a.op]
    sv = synth.lsrtm(nt=a.nt)
    wav = sv.wavelet()
    with Context(0) as ctx, Plan(ctx, op, sv.shots) as p:
        if op != OP_BORN_ADJOINT:
            p.set_exact(a.exact)
        for i in range(len(sv.shots)):
            p.set(i, IN_VEL, sv.sub(sv.vel0, i))
            p.set(i, IN_WAVELET, wav)
            if op == OP_BORN:
                p.set(i, IN_DV, sv.sub(sv.dv, i))
        ms, by = p.time_kernels(a.steps)
    print(json.dumps({"op": a.op, "interior_ms": ms[0], "pad_ms": ms[1], "step_ms": ms[2],
                      "interior_bytes": by[0], "pad_bytes": by[1]}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
