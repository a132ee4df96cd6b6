import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "graph-bit-ops_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# the reference checkout (GBO_REF_DIR), present only where it is mounted
REF_ROOT = os.environ.get("GBO_REF_DIR", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def gbo():
    import gbo as m

    m.lib()  # raises if libgbo.so is missing: no silent fallback
    return m


@pytest.fixture(scope="session")
def orc():
    import oracle as m

    m.lib()
    return m


@pytest.fixture(scope="session")
def gpu(gbo):
    n = gbo.device_count()
    assert n > 0, "GPU test collected but no CUDA device is visible"
    gbo.check(gbo.lib().gbo_set_device(0))
    return 0


def ref_path(rel):
    p = os.path.join(REF_ROOT, rel)
    return p if os.path.exists(p) else None


def sha(a) -> str:
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]
