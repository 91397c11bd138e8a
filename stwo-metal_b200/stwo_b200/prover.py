"""Wide-Fibonacci proving on the B200 (stwo::prover::prove for the
Wide-Fibonacci component, crates/stwo/src/prover/mod.rs:32-138)."""
from __future__ import annotations

import ctypes as C

from . import ffi
from .backend import DeviceColumn, as_stream


class WideFibConfig(C.Structure):
    """PcsConfig / FriConfig fields (crates/stwo/src/core/pcs/mod.rs:31-80)."""
    _fields_ = [("log_n_rows", C.c_uint32), ("n_cols", C.c_uint32), ("log_blowup", C.c_uint32),
                ("pow_bits", C.c_uint32), ("n_queries", C.c_uint32), ("log_last_layer_degree_bound", C.c_uint32),
                ("line_fold_step", C.c_uint32), ("m31_channel", C.c_int32)]


def wide_fib_config(log_n_rows: int, n_cols: int = 100, log_blowup: int = 1, pow_bits: int = 10, n_queries: int = 3,
                    log_last_layer_degree_bound: int = 0, line_fold_step: int = 1,
                    m31_channel: bool = False) -> WideFibConfig:
    return WideFibConfig(log_n_rows, n_cols, log_blowup, pow_bits, n_queries, log_last_layer_degree_bound,
                         line_fold_step, int(m31_channel))


class WideFibProver:
    """Owns the device buffers of one proof shape; proves repeatedly."""

    def __init__(self, cfg: WideFibConfig, stream=None):
        ffi.init()
        self.cfg = cfg
        self.stream = as_stream(stream)
        h = C.c_void_p()
        ffi.call("stwo_b200_prover_create", C.byref(cfg), C.byref(h), self.stream)
        self.handle = h

    def prove(self, a: DeviceColumn, b: DeviceColumn, cap: int = 1 << 22) -> bytes:
        buf = (C.c_uint8 * cap)()
        n = C.c_size_t()
        ffi.call("stwo_b200_prove_wide_fib", self.handle, C.c_void_p(a.ptr), C.c_void_p(b.ptr), buf,
                 C.c_size_t(cap), C.byref(n))
        return bytes(buf[:n.value])

    def prove_into(self, a_ptr: int, b_ptr: int, out_buf, cap: int) -> int:
        n = C.c_size_t()
        ffi.call("stwo_b200_prove_wide_fib", self.handle, C.c_void_p(a_ptr), C.c_void_p(b_ptr), out_buf,
                 C.c_size_t(cap), C.byref(n))
        return n.value

    def close(self):
        if getattr(self, "handle", None):
            ffi.call("stwo_b200_prover_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
