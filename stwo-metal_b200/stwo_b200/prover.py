"""Wide-Fibonacci proving on the B200 (stwo::prover::prove for the
Wide-Fibonacci component, crates/stwo/src/prover/mod.rs:32-138)."""
from __future__ import annotations

import ctypes as C

import numpy as np

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
        return C.string_at(buf, n.value)

    def prove_cols(self, a: DeviceColumn, b: DeviceColumn, n_cols: int, cap: int = 1 << 22) -> bytes:
        """The proof of an n_cols-wide trace (3 <= n_cols <= the prover's width)."""
        buf = (C.c_uint8 * cap)()
        n = C.c_size_t()
        ffi.call("stwo_b200_prove_wide_fib_cols", self.handle, C.c_uint32(n_cols), C.c_void_p(a.ptr),
                 C.c_void_p(b.ptr), buf, C.c_size_t(cap), C.byref(n))
        return C.string_at(buf, n.value)

    def prove_host(self, a: np.ndarray, b: np.ndarray, cap: int = 1 << 22) -> bytes:
        """The proof from host columns (numpy, uint32); copied by the prover,
        overlapped with the trace generation when the memory is pinned."""
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = np.ascontiguousarray(b, dtype=np.uint32)
        buf = (C.c_uint8 * cap)()
        n = C.c_size_t()
        ffi.call("stwo_b200_prove_wide_fib_host", self.handle, C.c_void_p(a.ctypes.data), C.c_void_p(b.ctypes.data),
                 buf, C.c_size_t(cap), C.byref(n))
        return C.string_at(buf, n.value)

    def prove_host_into(self, a_ptr: int, b_ptr: int, out_buf, cap: int) -> int:
        """prove_host from raw host pointers (e.g. pinned buffers) into out_buf."""
        n = C.c_size_t()
        ffi.call("stwo_b200_prove_wide_fib_host", self.handle, C.c_void_p(a_ptr), C.c_void_p(b_ptr), out_buf,
                 C.c_size_t(cap), C.byref(n))
        return n.value

    def prove_into(self, a_ptr: int, b_ptr: int, out_buf, cap: int) -> int:
        n = C.c_size_t()
        ffi.call("stwo_b200_prove_wide_fib", self.handle, C.c_void_p(a_ptr), C.c_void_p(b_ptr), out_buf,
                 C.c_size_t(cap), C.byref(n))
        return n.value

    STREAM_SPIN_DEFAULT = 1 << 22

    def set_stream_spin(self, polls: int) -> None:
        """Poll bound of a consumer's stage wait in the column-streaming
        kernels (composition, quotients); 0 makes every such wait give up at
        once, so the prove returns STWO_B200_ETIMEOUT."""
        ffi.call("stwo_b200_prover_set_stream_spin", self.handle, C.c_uint32(polls))

    def close(self):
        if getattr(self, "handle", None):
            ffi.call("stwo_b200_prover_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SeededFriProver:
    """FriProver commit + decommit of one secure column with supplied alphas
    (crates/stwo/src/prover/fri.rs:133-350): every layer folded by 2 down to one
    value, a Blake2s tree per layer, the queried decommitments.  ``prove``
    returns the FriProof bytes in the proof's canonical layout."""

    def __init__(self, log_size: int, tree, m31: bool = False, stream=None):
        ffi.init()
        self.log_size = log_size
        self.stream = as_stream(stream)
        self._tree = tree  # the library keeps its device pointers: keep the buffers alive
        h = C.c_void_p()
        ffi.call("stwo_b200_fri_prover_create", C.c_uint32(log_size), C.c_int(1 if m31 else 0),
                 C.c_void_p(tree.itwiddles.ptr), C.c_uint32(tree.log_size), self.stream, C.byref(h))
        self._h = h

    def prove(self, coords, alphas, queries, cap: int = 1 << 22) -> bytes:
        a = np.ascontiguousarray(alphas, dtype=np.uint32).reshape(-1)
        q = np.ascontiguousarray(queries, dtype=np.uint64)
        ptrs = (C.c_void_p * 4)(*[c.ptr for c in coords])
        if getattr(self, "_buf", None) is None or len(self._buf) < cap:
            self._buf = (C.c_uint8 * cap)()  # reused across calls (a fresh one is zero-filled)
        buf = self._buf
        n = C.c_size_t()
        ffi.call("stwo_b200_fri_prove_seeded", self._h, ptrs, a.ctypes.data_as(C.POINTER(C.c_uint32)),
                 q.ctypes.data_as(C.POINTER(C.c_uint64)), C.c_uint32(q.size), buf, C.c_size_t(len(buf)),
                 C.byref(n))
        return C.string_at(buf, n.value)

    def close(self):
        if self._h:
            ffi.call("stwo_b200_fri_prover_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def prover_footprint(cfg: WideFibConfig) -> int:
    """Device bytes a prover of this configuration allocates (host-only query)."""
    n = C.c_size_t()
    ffi.call("stwo_b200_prover_footprint", C.byref(cfg), C.byref(n))
    return n.value


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("provers_created", C.c_uint64), ("provers_reused", C.c_uint64),
                ("provers_evicted", C.c_uint64), ("resident_bytes", C.c_uint64), ("residents", C.c_uint32),
                ("max_running", C.c_uint32), ("queued", C.c_uint32), ("pad", C.c_uint32)]


class ProveServer:
    """Continuous batching of Wide-Fibonacci prove requests on the current GPU:
    ``slots`` requests run at once on resident provers (kept per log size and
    width class), admitted under an HBM budget with LRU eviction of idle
    provers.  ``submit`` copies the inputs and returns a ticket; ``wait``
    returns (proof bytes, {queued_ms, service_ms, latency_ms})."""

    def __init__(self, hbm_budget_bytes: int, slots: int = 3):
        ffi.init()
        h = C.c_void_p()
        ffi.call("stwo_b200_server_create", C.c_size_t(hbm_budget_bytes), C.c_uint32(slots), C.byref(h))
        self._h = h

    def submit(self, cfg: WideFibConfig, a, b) -> int:
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = np.ascontiguousarray(b, dtype=np.uint32)
        assert a.size == b.size == 1 << cfg.log_n_rows
        t = C.c_uint64()
        ffi.call("stwo_b200_server_submit", self._h, C.byref(cfg), a.ctypes.data_as(C.POINTER(C.c_uint32)),
                 b.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(t))
        return t.value

    def wait(self, ticket: int, cap: int = 1 << 22):
        buf = C.create_string_buffer(cap)
        n = C.c_size_t()
        times = (C.c_double * 3)()
        ffi.call("stwo_b200_server_wait", self._h, C.c_uint64(ticket), buf, C.c_size_t(cap), C.byref(n), times)
        return C.string_at(buf, n.value), {"queued_ms": times[0], "service_ms": times[1], "latency_ms": times[2]}

    def stats(self) -> dict:
        st = ServerStats()
        ffi.call("stwo_b200_server_get_stats", self._h, C.byref(st))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_ if k != "pad"}

    def close(self):
        if self._h:
            ffi.call("stwo_b200_server_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
