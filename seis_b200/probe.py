"""Per-kernel timing of one operator's step kernels on the LSRTM survey
(32 shots, 1200 x 400 model): the program the profiles under profiles/ are
captured from.

    python -m seis_b200.probe {born|modeling|adjoint} [--steps K] [--nt NT] [--exact]

Prints the interior-tile, pad-path and whole-step milliseconds (CUDA events,
kernels concurrent as in a run) and the algorithmic bytes of each.
"""
from __future__ import annotations

import argparse
import json


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m seis_b200.probe")
    ap.add_argument("op", choices=["born", "modeling", "adjoint"])
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--nt", type=int, default=400)
    ap.add_argument("--exact", action="store_true")
    a = ap.parse_args(argv)
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
