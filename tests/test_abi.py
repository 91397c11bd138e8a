"""The C-ABI library loads and exports every symbol include/stwo_b200.h
declares (no GPU needed: nothing is called)."""
import ctypes
import pytest

from stwo_b200 import ffi


def test_library_builds_and_loads():
    lib = ffi.load()
    assert "sm_100a" in ffi.version()
    assert lib is not None


def test_every_declared_symbol_is_exported():
    names = ffi.declared_symbols()
    assert len(names) >= 20
    lib = ffi.load()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_init_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(ffi.B200Error):
        ffi.call("stwo_b200_init", ctypes.c_int(0))


def test_integration_binding_declares_every_entry_point():
    # the Rust extern block a maintainer adds covers the whole header
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    text = open(os.path.join(root, "INTEGRATION.md")).read()
    bound = set(re.findall(r"pub fn (stwo_b200_[a-z0-9_]+)\s*\(", text))
    missing = [n for n in ffi.declared_symbols() if n not in bound]
    assert not missing, missing
