"""ctypes binding of ``libstwo_b200.so`` (the sm_100a kernels + C ABI).

Every C entry point returns 0 or a negative status and writes a message into a
caller buffer; :func:`call` turns failures into :class:`B200Error`.  There is
no CPU fallback: loading fails loudly when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_ROOT, "libstwo_b200.so")
HEADER = os.path.join(os.path.dirname(PKG_ROOT), "include", "stwo_b200.h")

_lib = None
_initialized = False


class B200Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"stwo_b200 error {code}: {msg}")
        self.code = code


def load(build_if_missing: bool = True):
    """Loads the shared library (building it with nvcc if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            if not build_if_missing:
                raise B200Error(-5, f"{LIB_PATH} not built")
            import importlib.util
            spec = importlib.util.spec_from_file_location("stwo_b200_build", os.path.join(PKG_ROOT, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        _lib = C.CDLL(LIB_PATH)
        _lib.stwo_b200_version.restype = C.c_char_p
        _lib.stwo_b200_launch_count.restype = C.c_uint64
    return _lib


def declared_symbols() -> list[str]:
    """Function names declared in include/stwo_b200.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(stwo_b200_[a-z0-9_]+)\s*\(", text)))


def call(fn_name: str, *args) -> None:
    err = C.create_string_buffer(512)
    rc = getattr(load(), fn_name)(*args, err, C.c_size_t(len(err)))
    if rc != 0:
        raise B200Error(rc, err.value.decode(errors="replace"))


def init(device: int = 0) -> None:
    """Selects the device; raises when no sm_100 GPU is present."""
    global _initialized
    if not _initialized:
        call("stwo_b200_init", C.c_int(device))
        _initialized = True


def launch_count() -> int:
    """Kernels launched by libstwo_b200 so far (host-side counter)."""
    return int(load().stwo_b200_launch_count())


def version() -> str:
    return load().stwo_b200_version().decode()
