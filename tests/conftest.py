"""Shared fixtures.  `-m "not gpu"` runs on any CPU box; `-m gpu` needs a B200
and the in-tree libdimgpu.so."""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built libdimgpu.so")
    config.addinivalue_line("markers", "slow: long CPU stress tests, run only when selected with -m slow")


def pytest_collection_modifyitems(config, items):
    """`slow` tests are opt-in: they run only when the -m expression names them."""
    if "slow" in (config.getoption("-m") or ""):
        return
    skip = pytest.mark.skip(reason="opt-in: select with -m slow")
    for item in items:
        if "slow" in item.keywords:
            item.add_marker(skip)


HOST_SO = os.path.join(ROOT, "tests", "_build", "libphyshost.so")


def build_host_harness() -> str:
    """g++ build of the device arithmetic for the host (tests/native)."""
    src = os.path.join(ROOT, "tests", "native", "physics_host.cpp")
    csrc = os.path.join(ROOT, "diffuse_vs_gfm_mms_b200", "csrc")
    deps = [src] + [os.path.join(csrc, h) for h in ("dim_physics.h", "dim_line.h", "dim_mixed.h",
                                                                "euler_physics.h", "fastdiv.h")]
    if os.path.exists(HOST_SO) and os.path.getmtime(HOST_SO) >= max(os.path.getmtime(p) for p in deps):
        return HOST_SO
    os.makedirs(os.path.dirname(HOST_SO), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", f"-I{os.path.join(ROOT, 'include')}", src,
           "-o", HOST_SO]
    subprocess.run(cmd, check=True)
    return HOST_SO


@pytest.fixture(scope="session")
def port():
    from oracle import oracle as O
    if not os.path.exists(O.PORT_SO):
        O.build()
    return O.port()


@pytest.fixture(scope="session")
def reference():
    from oracle import oracle as O
    if not O.reference_available():
        pytest.skip("reference build (oracle/_ref) absent")
    return O.reference()


@pytest.fixture(scope="session")
def euler_port():
    from oracle import oracle as O
    if not os.path.exists(O.PORT_SO):
        O.build()
    return O.EulerChecker("port")


@pytest.fixture(scope="session")
def euler_reference():
    from oracle import oracle as O
    if not os.path.exists(O.EREF_SO):
        pytest.skip("reference Euler build (oracle/_ref/libeulerref.so) absent")
    return O.EulerChecker("reference")
