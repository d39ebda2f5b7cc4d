"""The C ABI library loads and exports every entry point include/pdem.h declares (no GPU work)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pdem.h")
LIB = os.path.join(ROOT, "peclet-dem_b200", "peclet", "dem", "libpdem.so")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pdem_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "pdem_create" in names and "pdem_step" in names and "pdem_step_hertz" in names
    assert len(names) >= 60


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"


def test_python_binding_covers_the_abi():
    from peclet.dem import _capi
    names = {f"pdem_{k}" for k in _capi._SIGS}
    missing = [n for n in declared() if n not in names and n != "pdem_execution_space"]
    assert not missing, f"ABI entry points without a binding: {missing}"


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        return
    import peclet.dem as dem
    import pytest
    with pytest.raises(RuntimeError, match="CUDA"):
        dem.Simulation(16)
