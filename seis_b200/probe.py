"""Measurement programs.

    python -m seis_b200.probe {born|modeling|adjoint} [--steps K] [--nt NT] [--exact]

Per-kernel timing of one operator's step kernels on the LSRTM survey (32
shots, 1200 x 400 model): the program the profiles under profiles/ are
captured from.  Prints the interior-tile, pad-path and whole-step milliseconds
(CUDA events, kernels concurrent as in a run) and the algorithmic bytes of
each.

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


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m seis_b200.probe")
    ap.add_argument("op", choices=["born", "modeling", "adjoint", "snapshots"])
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--nt", type=int, default=None,
                    help="time samples (default 400; snapshots: 4000)")
    ap.add_argument("--exact", action="store_true")
    a = ap.parse_args(argv)
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
