"""Test configuration: markers, import paths and the test-only checkers.

`-m gpu` tests need a CUDA device and call the B200 library through its C ABI; everything else runs
on the CPU. The oracle restatement (oracle/restate) is built on demand with g++; the reference build
(oracle/_ref, compiled from the reference sources against the Kokkos shim) is used when present.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "peclet-dem_b200")
for p in (PKG, os.path.join(ROOT, "tests"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

ORC_LIB = os.path.join(ROOT, "oracle", "_build", "liborc.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_serial.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the C ABI")


def _build_oracle():
    # make rebuilds only what is stale; without g++ (a box that only runs prebuilt files) the
    # library already there is used
    try:
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "orc"], check=True)
    except (OSError, subprocess.CalledProcessError):
        if not os.path.exists(ORC_LIB):
            raise
    return ORC_LIB


@pytest.fixture(scope="session")
def orc_api():
    from peclet.dem._capi import CApi
    return CApi(_build_oracle(), "orc")


@pytest.fixture(scope="session")
def ref_api():
    from peclet.dem._capi import CApi
    if not os.path.exists(REF_LIB):
        pytest.skip("reference build (oracle/_ref) not present")
    return CApi(REF_LIB, "ref")


@pytest.fixture(scope="session")
def gpu_api():
    import ctypes
    try:
        import peclet.dem as dem
    except ImportError as e:
        pytest.fail(f"B200 library missing: {e}")
    h = ctypes.c_void_p()
    st = dem._API.fn["create"](16, 64, ctypes.byref(h))
    if st != 0:
        pytest.fail(f"no usable CUDA device: {dem._API.error()}")
    dem._API.fn["destroy"](h)
    return dem._API
