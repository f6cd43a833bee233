import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: full-size workload")
    lib = os.path.join(ROOT, "seis_b200", "lib", "libseisfd.so")
    if not os.path.exists(lib):  # nvcc cross-compiles without a device
        subprocess.run([sys.executable, "-m", "seis_b200.build"], cwd=ROOT, check=True,
                       capture_output=True)
    so = os.path.join(ROOT, "oracle", "_build", "libseisoracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "_build/libseisoracle.so"],
                       check=True, capture_output=True)


@pytest.fixture(scope="session")
def ctx():
    import seis_b200
    c = seis_b200.Context(0)
    yield c
    c.close()
