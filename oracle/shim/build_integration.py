"""Build oracle/_ref/fd_shim_check: the fd.h drop-in printed in INTEGRATION.md,
compiled as written against the reference's own src/util/fd.h and memory.h,
and linked with the reference's callers (src/lsrtm/inversion.cpp, whose
Inversion::modeling_MPI, forward_MPI, adjoint_MPI, illum_MPI, illumPlane_MPI
and plane-wave members call modeling / forward / adjoint / illum /
illumPlane / forwordPlane / adjointPlane) and with libseisfd.so.  Test
infrastructure only.

The reference's own versions of the drop-in's functions are made local to
their object file (objcopy --localize-symbol), so every call from the
reference's callers must bind to the drop-in: a signature that differs from
fd.h's leaves an undefined symbol and the link fails.  The harness
(fd_shim_harness.cpp) runs the drop-in functions on one shot read from a file
(tests/test_gpu_integration.py).

    python oracle/shim/build_integration.py REF   (from oracle/Makefile)
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

SHIM = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(SHIM)
ROOT = os.path.dirname(ORACLE)
OUT = os.path.join(ORACLE, "_ref")
API = ["modeling", "forward", "adjoint", "adjointUpDown", "forwordPlane", "adjointPlane",
       "rtm_true", "illum", "illumPlane"]
OTHER_SRC = ["util/InitInversion.cpp", "util/global.cpp", "util/wavelet.cpp", "util/parser.cpp",
             "util/coord.cpp", "lsrtm/datastr.cpp", "filter/smooth.cpp", "util/io.cpp"]


def extract(md_path: str) -> str:
    """The C++ blocks of INTEGRATION.md's fd.h drop-in section, in order."""
    text = open(md_path).read()
    start = text.index("## C++: a drop-in for `src/util/fd.h`")
    end = text.index("\n## ", start + 1)
    blocks = re.findall(r"```c\+\+\n(.*?)```", text[start:end], flags=re.S)
    if len(blocks) < 2:
        raise SystemExit("INTEGRATION.md: expected the two drop-in code blocks")
    return "// extracted from INTEGRATION.md by oracle/shim/build_integration.py\n" + "\n".join(blocks)


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise SystemExit(f"step failed: {cmd[0]}")
    return r.stdout


def build(ref: str, source: str, out_dir: str = OUT) -> str:
    """Compile `source` (the drop-in) with the harness, the reference's
    callers and libseisfd.so into out_dir/fd_shim_check; raises SystemExit
    if a step fails (a link error when a drop-in signature differs from
    fd.h's)."""
    os.makedirs(out_dir, exist_ok=True)
    src = os.path.join(out_dir, "fd_gpu.cpp")
    open(src, "w").write(source)
    base = ["g++", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-std=c++11", "-fpermissive",
            "-w", "-include", os.path.join(SHIM, "ref_shim.h"),
            f"-I{ref}/src/util", f"-I{ref}/src/filter", f"-I{ref}/src/lsrtm", f"-I{SHIM}"]
    fd_o, fd_local = os.path.join(out_dir, "fd_plain.o"), os.path.join(out_dir, "fd_local.o")
    run(base + ["-c", "-o", fd_o, f"{ref}/src/util/fd.cpp"])
    syms = []
    for line in run(["nm", "-g", "--defined-only", fd_o]).splitlines():
        name = line.split()[-1]
        if run(["c++filt", name]).strip().split("(")[0] in API:
            syms.append(name)
    if len(syms) != len(API):
        raise SystemExit(f"fd.o: found {len(syms)} of the {len(API)} drop-in functions")
    run(["objcopy"] + [f"--localize-symbol={s}" for s in syms] + [fd_o, fd_local])
    exe = os.path.join(out_dir, "fd_shim_check")
    lib_dir = os.path.join(ROOT, "seis_b200", "lib")
    rpath = os.path.relpath(lib_dir, out_dir)
    run(base + [f"-I{ROOT}/include", "-o", exe, src, os.path.join(SHIM, "fd_shim_harness.cpp"),
                fd_local, os.path.join(OUT, "inversion.o"), os.path.join(SHIM, "ref_shim.cpp")]
        + [f"{ref}/src/{p}" for p in OTHER_SRC]
        + [f"-L{lib_dir}", "-lseisfd", f"-Wl,-rpath,$ORIGIN/{rpath}"])
    return exe


if __name__ == "__main__":
    print(build(sys.argv[1], extract(os.path.join(ROOT, "INTEGRATION.md"))))
