import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_oracle():
    so = os.path.join(ROOT, "oracle", "liboracle.so")
    src = os.path.join(ROOT, "oracle", "xnyz_oracle.cpp")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["bash", os.path.join(ROOT, "oracle", "build_oracle.sh")], check=True, capture_output=True)


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, available_reference
    if not available_reference():
        pytest.skip("the reference was not built here (oracle/_ref)")
    r = Reference()
    return r


@pytest.fixture(scope="session")
def xnyz():
    import xnyzip_b200
    return xnyzip_b200


@pytest.fixture(scope="session")
def ctx(xnyz):
    c = xnyz.Context(0)
    yield c
    c.close()


def quiet_call(reference, fn, *a, **k):
    """Run a reference call with its stdout chatter redirected."""
    reference.quiet(True)
    try:
        return fn(*a, **k)
    finally:
        reference.quiet(False)


# Small matrix of inputs shared by the CPU and GPU parity tests: (name, generator).
def small_inputs(n=4000):
    from xnyzip_b200 import synthetic as S
    return {
        "uniform": S.uniform(n, 3),
        "small_extent": np.random.default_rng(5).uniform(0, 3, (n, 3)).astype(np.float32),
        "duplicates": S.with_duplicates(n, 4),
        "planar": S.planar(n, 6),
        "terrain": S.terrain(n, 7, extent=300.0, amplitude=3.0, wavelength=150.0),
        "spheres": S.spheres(n, 20, 8, extent=400.0),
    }
