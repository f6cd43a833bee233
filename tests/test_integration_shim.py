"""INTEGRATION.md's drop-in for the reference's src/util/fd.h, compiled as
printed against the reference's own fd.h and memory.h and linked with the
reference's callers (src/lsrtm/inversion.cpp) and libseisfd.so
(oracle/shim/build_integration.py).  Host-only: building needs the reference
checkout, running it is tests/test_gpu_integration.py."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle", "shim"))
import build_integration as B  # noqa: E402

REF = os.environ.get("SEIS_REFERENCE_DIR", "/root/reference")
need_ref = pytest.mark.skipif(
    not os.path.isfile(os.path.join(REF, "src", "util", "fd.cpp"))
    or not os.path.isfile(os.path.join(ROOT, "oracle", "_ref", "inversion.o")),
    reason="reference checkout or its compiled callers absent")


@need_ref
def test_drop_in_builds_and_binds_every_caller(tmp_path):
    src = B.extract(os.path.join(ROOT, "INTEGRATION.md"))
    for name in B.API:  # every fd.h function a caller can reach is defined
        assert f"float **{name}(" in src, name
    exe = B.build(REF, src, str(tmp_path))
    assert os.access(exe, os.X_OK)


@need_ref
def test_a_signature_that_differs_from_fd_h_fails_to_link(tmp_path):
    """The check has teeth: with `modeling` taking a double time step, the
    reference's Inversion::modeling_MPI call has nothing to bind to."""
    src = B.extract(os.path.join(ROOT, "INTEGRATION.md"))
    bad = src.replace("float **modeling(float dt,", "float **modeling(double dt,", 1)
    assert bad != src
    with pytest.raises(SystemExit):
        B.build(REF, bad, str(tmp_path))
