import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PACKAGE = os.path.join(ROOT, "global-illumination_b200")
sys.path.insert(0, PACKAGE)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


def _ensure_built():
    if not os.path.exists(os.path.join(PACKAGE, "libvgi.so")):
        subprocess.run(["make", "-s", "-C", PACKAGE, "-j4"], check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def gpu():
    """A libvgi context on cuda:0 (the tests marked gpu use it)."""
    import vgi

    tracer = vgi.GpuTracer(0)
    yield tracer
    tracer.close()
