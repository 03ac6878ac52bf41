import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")

# The reference checkout, for the CPU tests that read its sources: the
# MBX_REFERENCE environment variable, else the build machine's checkout when
# present (GPU machines have none; those tests skip or use the fixtures).
if not os.environ.get("MBX_REFERENCE") and os.path.isdir("/root/reference/src"):
    os.environ["MBX_REFERENCE"] = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


def pytest_sessionstart(session):
    """The compiled reference (oracle/_ref) is the oracle of many CPU tests:
    build it on demand where its sources are present and it is not built yet
    (a few minutes, once)."""
    import subprocess
    ref = os.environ.get("MBX_REFERENCE")
    lib = os.path.join(ROOT, "oracle", "_ref", "libmbx_ref.so")
    if ref and os.path.isdir(os.path.join(ref, "src")) and not os.path.exists(lib):
        subprocess.call([sys.executable, os.path.join(ROOT, "oracle", "build_ref.py"), "--ref", ref])


def golden(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        return json.load(f)


def has_ref():
    import mbx_oracle
    return mbx_oracle.RefSystem.available()


@pytest.fixture(scope="session")
def ctx():
    from mbx_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()


# GPU suite order: the path itself first (evaluator goldens, boxes against the
# reference, lists), then batching and the autograd wrapper; the
# allocation-free entry point (tests/test_zz_no_alloc.py) stays last.  A run
# that stops at the first failure has then checked the path before anything
# built on it.
_ORDER = ("test_capi_load", "test_gpu_parity", "test_gpu_batch", "test_gpu_autograd", "test_cxx_boundary")


def pytest_collection_modifyitems(session, config, items):
    def rank(item):
        mod = item.module.__name__.rsplit(".", 1)[-1]
        if mod.startswith("test_zz"):
            return len(_ORDER) + 1
        return _ORDER.index(mod) if mod in _ORDER else len(_ORDER)
    items.sort(key=rank)   # stable: keeps the order within a file
