"""Build ``seis_b200/lib/libseisfd.so`` (the C-ABI library) in-tree with nvcc.

The CUDA sources are compiled for sm_100a only, with ``--fmad=false`` and IEEE
division/square root so that the kernels round every operation on its own, as
the reference's x86-64 build does.  Host C++ is compiled with
``-ffp-contract=off`` for the same reason.

Usage: ``python -m seis_b200.build [--force]``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
OBJ_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libseisfd.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
               "-Xptxas", "-warn-spills"]
# exact flavour: every operation rounds on its own, IEEE division and sqrt
NVCC_EXACT = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"]
# fast flavour (sources named *_fast.cu): contraction and approximate division,
# denormals still kept (the decaying wavefield lives there)
NVCC_FAST = ["--fmad=true", "-prec-div=false", "-prec-sqrt=false"]
# accurate flavour (sources named *_acc.cu): contraction, IEEE division / sqrt
NVCC_ACC = ["--fmad=true", "-prec-div=true", "-prec-sqrt=true"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function"]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _cuda_include():
    return os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


def _sources():
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return [os.path.join(CSRC, s) for s in srcs], headers


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs, headers = _sources()
    nvcc = _nvcc()
    objs, cmds = [], []
    for src in srcs:
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src] + headers + [__file__]):
            continue
        if src.endswith(".cu"):
            flav = (NVCC_FAST if src.endswith("_fast.cu")
                    else NVCC_ACC if src.endswith("_acc.cu") else NVCC_EXACT)
            cmd = [nvcc, *ARCH, *NVCC_COMMON, *flav, "-I", CSRC, "-I", INCLUDE, "-c", "-o", obj, src]
        else:
            cmd = ["g++", *CXX_FLAGS, "-I", CSRC, "-I", INCLUDE, "-I", _cuda_include(), "-c", "-o", obj, src]
        cmds.append(cmd)
    # translation units compile independently (the step kernels of every tile
    # shape make the CUDA ones the slow part)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for out in ex.map(_run, cmds):
            if verbose and out.strip():
                sys.stderr.write(out)
    if force or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
