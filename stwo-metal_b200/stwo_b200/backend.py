"""Python view of the B200 backend: device columns and stwo's Backend ops.

Mirrors the trait surface of ``crates/stwo/src/prover/backend/mod.rs`` (ColumnOps,
PolyOps, MerkleOpsLifted, MerkleOps, FriOps) over the C ABI in
``include/stwo_b200.h``.  Columns live in device memory (:class:`DeviceColumn`);
host copies happen only through :meth:`DeviceColumn.from_host` /
:meth:`DeviceColumn.to_host`.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import ffi

P = (1 << 31) - 1


def as_stream(stream):
    """cudaStream_t for ctypes: None (legacy default stream), an int handle
    (e.g. torch.cuda.Stream().cuda_stream) or a c_void_p."""
    if stream is None or isinstance(stream, C.c_void_p):
        return stream
    return C.c_void_p(int(stream))


class DeviceBuffer:
    """Device memory from the stream-ordered pool; freed on close()/GC."""

    def __init__(self, nbytes: int, stream=None):
        ffi.init()
        self.nbytes = int(nbytes)
        stream = as_stream(stream)
        self.stream = stream
        ptr = C.c_void_p()
        ffi.call("stwo_b200_alloc", C.c_size_t(self.nbytes), C.byref(ptr), stream)
        self.ptr = ptr.value or 0

    def close(self):
        if getattr(self, "ptr", 0):
            ffi.call("stwo_b200_free", C.c_void_p(self.ptr), self.stream)
            self.ptr = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, host: np.ndarray, offset: int = 0):
        host = np.ascontiguousarray(host)
        assert offset + host.nbytes <= self.nbytes
        ffi.call("stwo_b200_memcpy_h2d", C.c_void_p(self.ptr + offset), host.ctypes.data_as(C.c_void_p),
                 C.c_size_t(host.nbytes), self.stream)
        sync(self.stream)

    def download(self, dtype=np.uint32, count=None, offset: int = 0) -> np.ndarray:
        dtype = np.dtype(dtype)
        if count is None:
            count = (self.nbytes - offset) // dtype.itemsize
        out = np.empty(count, dtype)
        ffi.call("stwo_b200_memcpy_d2h", out.ctypes.data_as(C.c_void_p), C.c_void_p(self.ptr + offset),
                 C.c_size_t(out.nbytes), self.stream)
        sync(self.stream)
        return out


def sync(stream=None):
    ffi.call("stwo_b200_stream_sync", as_stream(stream))


class DeviceColumn(DeviceBuffer):
    """A column of M31 words on the device (Col<B200Backend, BaseField>)."""

    def __init__(self, length: int, stream=None):
        super().__init__(4 * length, stream)
        self.length = int(length)

    @property
    def log_size(self) -> int:
        return self.length.bit_length() - 1

    @classmethod
    def from_host(cls, values, stream=None) -> "DeviceColumn":
        values = np.ascontiguousarray(values, dtype=np.uint32)
        col = cls(values.size, stream)
        if values.size:
            col.upload(values)
        return col

    def to_host(self) -> np.ndarray:
        return self.download(np.uint32, self.length)


class SecureColumn:
    """QM31 column as four M31 coordinate columns (SecureColumnByCoords)."""

    def __init__(self, cols):
        self.cols = list(cols)
        assert len(self.cols) == 4

    @classmethod
    def from_host(cls, coords, stream=None):
        return cls([DeviceColumn.from_host(c, stream) for c in coords])

    @classmethod
    def empty(cls, length, stream=None):
        return cls([DeviceColumn(length, stream) for _ in range(4)])

    def to_host(self):
        return [c.to_host() for c in self.cols]

    @property
    def length(self):
        return self.cols[0].length


@dataclass
class TwiddleTree:
    """PolyOps::Twiddles: tree of the root coset (canonical values)."""
    root_initial_index: int
    log_size: int
    twiddles: DeviceColumn
    itwiddles: DeviceColumn


def _ptr_array(cols):
    return (C.c_void_p * max(1, len(cols)))(*[c.ptr for c in cols])


def _u32_array(vals):
    return (C.c_uint32 * max(1, len(vals)))(*[int(v) for v in vals])


def canonic_half_coset(log_size: int):
    """(initial_index, log_size) of CanonicCoset(log_size).half_coset."""
    return 1 << (31 - (log_size + 1)), log_size - 1


class B200Backend:
    """The Backend trait surface on one B200 (all ops enqueue on `stream`)."""

    def __init__(self, stream=None):
        ffi.init()
        self.stream = as_stream(stream)

    # ---- PolyOps::precompute_twiddles --------------------------------------
    def precompute_twiddles(self, initial_index: int, log_size: int) -> TwiddleTree:
        tw = DeviceColumn(1 << log_size, self.stream)
        itw = DeviceColumn(1 << log_size, self.stream)
        ffi.call("stwo_b200_precompute_twiddles", C.c_uint64(initial_index), C.c_uint32(log_size),
                 C.c_void_p(tw.ptr), C.c_void_p(itw.ptr), self.stream)
        return TwiddleTree(initial_index, log_size, tw, itw)

    # ---- ColumnOps::bit_reverse_column --------------------------------------
    def bit_reverse_column(self, col: DeviceColumn):
        ffi.call("stwo_b200_bit_reverse_column", C.c_void_p(col.ptr), C.c_uint32(col.log_size), self.stream)

    def bit_reverse_columns(self, srcs, dsts=None):
        """bit_reverse_column over many columns in one call: into ``dsts``
        (same sizes), or in place when ``dsts`` is None."""
        dsts = srcs if dsts is None else dsts
        if len(dsts) != len(srcs) or any(d.log_size != s_.log_size for s_, d in zip(srcs, dsts)):
            raise ValueError("source and destination columns differ in number or size")
        ffi.call("stwo_b200_bit_reverse_columns", _ptr_array(srcs), _ptr_array(dsts),
                 _u32_array([c.log_size for c in srcs]), C.c_uint32(len(srcs)), self.stream)

    # ---- PolyOps::interpolate_columns (in place) ------------------------------
    def interpolate_columns(self, cols, tree: TwiddleTree, half_initial_indices=None):
        his = None
        if half_initial_indices is not None:
            his = (C.c_uint64 * len(cols))(*half_initial_indices)
        ffi.call("stwo_b200_interpolate_columns", _ptr_array(cols), _u32_array([c.log_size for c in cols]), his,
                 C.c_uint32(len(cols)), C.c_void_p(tree.itwiddles.ptr), C.c_uint32(tree.log_size), self.stream)
        return cols

    def interpolate_columns_into(self, evals, coeffs, tree: TwiddleTree):
        """Out-of-place interpolate: evals stay intact, coeffs receive the result."""
        ffi.call("stwo_b200_interpolate_columns_into", _ptr_array(evals), _ptr_array(coeffs),
                 _u32_array([c.log_size for c in evals]), None, C.c_uint32(len(evals)),
                 C.c_void_p(tree.itwiddles.ptr), C.c_uint32(tree.log_size), self.stream)
        return coeffs

    def interpolate_natural_into(self, naturals, coeffs, tree: TwiddleTree):
        """CircleEvaluation<NaturalOrder>::bit_reverse + interpolate in one call:
        natural-order evaluations in, coefficients out (the bit reversal rides
        on the first FFT pass where it can)."""
        if len(naturals) != len(coeffs) or any(a.log_size != b.log_size for a, b in zip(naturals, coeffs)):
            raise ValueError("source and destination columns differ in number or size")
        ffi.call("stwo_b200_interpolate_columns_natural", _ptr_array(naturals), _ptr_array(coeffs),
                 _u32_array([c.log_size for c in naturals]), None, C.c_uint32(len(naturals)),
                 C.c_void_p(tree.itwiddles.ptr), C.c_uint32(tree.log_size), self.stream)
        return coeffs

    def evaluate_polynomials_into(self, coeffs, log_blowup: int, tree: TwiddleTree, outs):
        ffi.call("stwo_b200_evaluate_polynomials", _ptr_array(coeffs), _u32_array([c.log_size for c in coeffs]),
                 C.c_uint32(len(coeffs)), C.c_uint32(log_blowup), _ptr_array(outs), C.c_void_p(tree.twiddles.ptr),
                 C.c_uint32(tree.log_size), self.stream)
        return outs

    def interpolate_evaluate_into(self, srcs, coeffs, log_blowup: int, tree: TwiddleTree, outs):
        """interpolate_columns + evaluate_polynomials of same-size columns in one
        call: srcs (evaluations, or None to transform coeffs in place) ->
        coeffs -> outs on the 2^log_blowup times larger domain."""
        log_size = coeffs[0].log_size if coeffs else 0
        ffi.call("stwo_b200_interpolate_evaluate_columns", _ptr_array(srcs) if srcs is not None else None,
                 _ptr_array(coeffs), _ptr_array(outs), C.c_uint32(len(coeffs)), C.c_uint32(log_size),
                 C.c_uint32(log_blowup), C.c_void_p(tree.itwiddles.ptr), C.c_void_p(tree.twiddles.ptr),
                 C.c_uint32(tree.log_size), self.stream)
        return outs

    # ---- PolyOps::evaluate_polynomials ---------------------------------------
    def evaluate_polynomials(self, coeffs, log_blowup: int, tree: TwiddleTree):
        outs = [DeviceColumn(c.length << log_blowup, self.stream) for c in coeffs]
        ffi.call("stwo_b200_evaluate_polynomials", _ptr_array(coeffs), _u32_array([c.log_size for c in coeffs]),
                 C.c_uint32(len(coeffs)), C.c_uint32(log_blowup), _ptr_array(outs), C.c_void_p(tree.twiddles.ptr),
                 C.c_uint32(tree.log_size), self.stream)
        return outs

    # ---- MerkleOpsLifted ----------------------------------------------------
    def build_leaves(self, cols, lifting_log_size: int, m31_output: bool = False) -> DeviceBuffer:
        n = (1 << lifting_log_size) if cols else 1
        out = DeviceBuffer(32 * n, self.stream)
        ffi.call("stwo_b200_merkle_build_leaves", _ptr_array(cols), _u32_array([c.log_size for c in cols]),
                 C.c_uint32(len(cols)), C.c_uint32(lifting_log_size), C.c_int(int(m31_output)), C.c_void_p(out.ptr),
                 self.stream)
        return out

    def build_next_layer(self, prev: DeviceBuffer, m31_output: bool = False) -> DeviceBuffer:
        n = prev.nbytes // 32
        out = DeviceBuffer(32 * (n // 2), self.stream)
        ffi.call("stwo_b200_merkle_build_next_layer", C.c_void_p(prev.ptr), C.c_uint32(n.bit_length() - 1),
                 C.c_int(int(m31_output)), C.c_void_p(out.ptr), self.stream)
        return out

    def build_merkle_layers(self, cols, lifting_log_size: int, m31_output: bool = False):
        """Layers root first: layers[k] holds 2^k hashes."""
        layers = [DeviceBuffer(32 << k, self.stream) for k in range(lifting_log_size + 1)]
        ffi.call("stwo_b200_merkle_build_layers", _ptr_array(cols), _u32_array([c.log_size for c in cols]),
                 C.c_uint32(len(cols)), C.c_uint32(lifting_log_size), C.c_int(int(m31_output)),
                 _ptr_array(layers), self.stream)
        return layers

    def build_leaves_layers(self, cols, lifting_log_size: int, layers, m31_output: bool = False):
        """Leaves of columns sorted by length into layers[L]; layers[k < L]
        hold the chaining values between the hashing stages until
        build_nodes overwrites them."""
        ffi.call("stwo_b200_merkle_build_leaves_layers", _ptr_array(cols), _u32_array([c.log_size for c in cols]),
                 C.c_uint32(len(cols)), C.c_uint32(lifting_log_size), C.c_int(int(m31_output)),
                 _ptr_array(layers), self.stream)
        return layers[lifting_log_size]

    def build_leaves_into(self, cols, lifting_log_size: int, out: DeviceBuffer, m31_output: bool = False):
        ffi.call("stwo_b200_merkle_build_leaves", _ptr_array(cols), _u32_array([c.log_size for c in cols]),
                 C.c_uint32(len(cols)), C.c_uint32(lifting_log_size), C.c_int(int(m31_output)), C.c_void_p(out.ptr),
                 self.stream)
        return out

    def build_nodes(self, layers, m31_output: bool = False):
        """Fills layers[L-1..0] from the leaves in layers[L]."""
        ffi.call("stwo_b200_merkle_build_nodes", _ptr_array(layers), C.c_uint32(len(layers) - 1),
                 C.c_int(int(m31_output)), self.stream)
        return layers

    # ---- MerkleOps::commit_on_layer ------------------------------------------
    def commit_on_layer(self, log_size: int, prev, cols, m31_output: bool = False) -> DeviceBuffer:
        out = DeviceBuffer(32 << log_size, self.stream)
        ffi.call("stwo_b200_commit_on_layer", C.c_uint32(log_size), C.c_void_p(prev.ptr if prev else 0),
                 _ptr_array(cols), C.c_uint32(len(cols)), C.c_int(int(m31_output)), C.c_void_p(out.ptr), self.stream)
        return out

    # ---- FriOps ---------------------------------------------------------------
    def fold_line(self, ev: SecureColumn, alpha, tree: TwiddleTree, fold_step: int = 1) -> SecureColumn:
        out = SecureColumn.empty(ev.length >> fold_step, self.stream)
        ffi.call("stwo_b200_fold_line", _ptr_array(ev.cols), C.c_uint32(ev.cols[0].log_size), _u32_array(alpha),
                 C.c_uint32(fold_step), C.c_void_p(tree.itwiddles.ptr), C.c_uint32(tree.log_size),
                 _ptr_array(out.cols), self.stream)
        return out

    def fold_circle_into_line(self, dst: SecureColumn, src: SecureColumn, alpha, tree: TwiddleTree,
                              half_initial_index=None):
        log_n = src.cols[0].log_size
        if half_initial_index is None:
            half_initial_index = canonic_half_coset(log_n)[0]
        ffi.call("stwo_b200_fold_circle_into_line", _ptr_array(dst.cols), _ptr_array(src.cols), C.c_uint32(log_n),
                 C.c_uint64(half_initial_index), _u32_array(alpha), C.c_void_p(tree.itwiddles.ptr),
                 C.c_uint32(tree.log_size), self.stream)
        return dst

    # ---- QuotientOps ----------------------------------------------------------
    def accumulate_numerators(self, cols, batches):
        """QuotientOps::accumulate_numerators over same-size columns; batches =
        [(point (8 words), [(column index, value (4), random coeff (4)), ...])].
        Returns [(partial numerator SecureColumn, first linear term (4,))]."""
        log_n = cols[0].log_size
        cb = (SampleBatch * max(1, len(batches)))()
        keep, outs = [], []
        for b, (point, terms) in enumerate(batches):
            arr = (NumeratorTerm * max(1, len(terms)))()
            for k, (idx, val, alpha) in enumerate(terms):
                arr[k].column_index = int(idx)
                arr[k].sample_value = _words(val, 4)
                arr[k].random_coeff = _words(alpha, 4)
            keep.append(arr)
            cb[b].point = _words(point, 8)
            cb[b].terms = C.cast(arr, C.POINTER(NumeratorTerm))
            cb[b].n_terms = len(terms)
            outs.append(SecureColumn.empty(1 << log_n, self.stream))
        first = (C.c_uint32 * (4 * max(1, len(batches))))()
        ffi.call("stwo_b200_accumulate_numerators", _ptr_array(cols), C.c_uint32(len(cols)), C.c_uint32(log_n), cb,
                 C.c_uint32(len(batches)), _ptr_array([c for o in outs for c in o.cols]), first, self.stream)
        return [(o, np.array(first[4 * b:4 * b + 4], np.uint32)) for b, o in enumerate(outs)]

    def compute_quotients_and_combine(self, accs, lifting_log_size: int) -> SecureColumn:
        """accs = [(point (8 words), partial numerator SecureColumn, first linear term (4))]."""
        arr = (AccumulatedNumeratorsC * max(1, len(accs)))()
        for z, (point, col, first) in enumerate(accs):
            arr[z].sample_point = _words(point, 8)
            arr[z].d_partial = (C.c_void_p * 4)(*[c.ptr for c in col.cols])
            arr[z].log_size = col.cols[0].log_size
            arr[z].first_linear_term = _words(first, 4)
        out = SecureColumn.empty(1 << lifting_log_size, self.stream)
        ffi.call("stwo_b200_compute_quotients_and_combine", arr, C.c_uint32(len(accs)), C.c_uint32(lifting_log_size),
                 _ptr_array(out.cols), self.stream)
        return out

    # ---- AccumulationOps --------------------------------------------------------
    def accumulate(self, col: SecureColumn, other: SecureColumn):
        ffi.call("stwo_b200_accumulate", _ptr_array(col.cols), _ptr_array(other.cols), C.c_uint64(col.length),
                 self.stream)
        return col

    def generate_secure_powers(self, felt, n: int) -> np.ndarray:
        buf = DeviceBuffer(16 * max(1, n), self.stream)
        ffi.call("stwo_b200_generate_secure_powers", _words(felt, 4), C.c_uint32(n), C.c_void_p(buf.ptr),
                 self.stream)
        return buf.download(np.uint32, 4 * n).reshape(n, 4)

    def lift_and_accumulate(self, cols, out: SecureColumn | None = None) -> SecureColumn:
        out = SecureColumn.empty(cols[-1].length, self.stream) if out is None else out
        ffi.call("stwo_b200_lift_and_accumulate", _ptr_array([c for sc in cols for c in sc.cols]),
                 _u32_array([sc.cols[0].log_size for sc in cols]), C.c_uint32(len(cols)), _ptr_array(out.cols),
                 self.stream)
        return out

    # ---- PolyOps::eval_at_point -----------------------------------------------
    def batch_eval_at_point(self, polys, point) -> np.ndarray:
        out = (C.c_uint32 * (4 * max(1, len(polys))))()
        ffi.call("stwo_b200_batch_eval_at_point", _ptr_array(polys), C.c_uint32(len(polys)),
                 C.c_uint32(polys[0].log_size if polys else 0), _words(point, 8), out, self.stream)
        return np.array(out[:4 * len(polys)], np.uint32).reshape(len(polys), 4)

    def eval_at_point(self, poly: DeviceColumn, point) -> np.ndarray:
        out = (C.c_uint32 * 4)()
        ffi.call("stwo_b200_eval_at_point", C.c_void_p(poly.ptr), C.c_uint32(poly.log_size), _words(point, 8), out,
                 self.stream)
        return np.array(out[:], np.uint32)

    # ---- GrindOps ---------------------------------------------------------------
    def grind(self, digest: bytes, pow_bits: int, m31_channel: bool = False) -> int:
        d = (C.c_uint8 * 32).from_buffer_copy(bytes(digest))
        nonce = C.c_uint64()
        ffi.call("stwo_b200_grind", d, C.c_uint32(pow_bits), C.c_int(int(m31_channel)), C.byref(nonce), self.stream)
        return nonce.value

    # ---- ColumnOps<SecureField> -------------------------------------------------
    def bit_reverse_secure_column(self, col: SecureColumn):
        ffi.call("stwo_b200_bit_reverse_secure_column", _ptr_array(col.cols), C.c_uint32(col.cols[0].log_size),
                 self.stream)
        return col

    def bit_reverse_secure_field(self, buf: DeviceBuffer, log_size: int):
        """In place, on QM31 values stored 4 words each."""
        ffi.call("stwo_b200_bit_reverse_secure_field", C.c_void_p(buf.ptr), C.c_uint32(log_size), self.stream)
        return buf

    def decompose(self, ev: SecureColumn):
        out = SecureColumn.empty(ev.length, self.stream)
        lam = (C.c_uint32 * 4)()
        ffi.call("stwo_b200_decompose", _ptr_array(ev.cols), C.c_uint32(ev.cols[0].log_size), _ptr_array(out.cols),
                 lam, self.stream)
        return out, np.array(list(lam), np.uint32)


# ---- C structures of the QuotientOps entry points ---------------------------
class NumeratorTerm(C.Structure):
    """stwo_b200_numerator_term (core/pcs/quotients.rs:63-71 NumeratorData)."""
    _fields_ = [("column_index", C.c_uint32), ("sample_value", C.c_uint32 * 4), ("random_coeff", C.c_uint32 * 4)]


class SampleBatch(C.Structure):
    """stwo_b200_sample_batch (core/pcs/quotients.rs:55-61 ColumnSampleBatch)."""
    _fields_ = [("point", C.c_uint32 * 8), ("terms", C.POINTER(NumeratorTerm)), ("n_terms", C.c_uint32)]


class AccumulatedNumeratorsC(C.Structure):
    """stwo_b200_accumulated_numerators (prover/pcs/quotient_ops.rs:48-74)."""
    _fields_ = [("sample_point", C.c_uint32 * 8), ("d_partial", C.c_void_p * 4), ("log_size", C.c_uint32),
                ("first_linear_term", C.c_uint32 * 4)]


def _words(v, n):
    a = np.asarray(v, dtype=np.uint32).reshape(-1)
    assert a.size == n
    return (C.c_uint32 * n)(*[int(x) for x in a])


def layer_to_host(buf: DeviceBuffer) -> np.ndarray:
    return buf.download(np.uint8).reshape(-1, 32)


# ---- FFT pass plans (the autotuner's knobs) ---------------------------------
def fft_set_plan(log_size: int, passes) -> None:
    """Process-wide pass plan of n-layer FFTs; ``passes=()`` restores the default."""
    passes = list(passes)
    ffi.call("stwo_b200_fft_set_plan", C.c_uint32(log_size), _u32_array(passes), C.c_uint32(len(passes)))


def fft_get_plan(log_size: int) -> list:
    buf = (C.c_uint32 * 4)()
    n = C.c_uint32(0)
    ffi.call("stwo_b200_fft_get_plan", C.c_uint32(log_size), buf, C.c_uint32(4), C.byref(n))
    return [int(buf[i]) for i in range(n.value)]


# ---- trace commitment --------------------------------------------------------
class Committer:
    """CommitmentTreeProver::new for one column set (crates/stwo/src/prover/pcs/
    mod.rs:707-781): interpolate, evaluate on the blowup domain, lifted Blake2s
    tree.  ``per_column`` launches every column on its own (the plain form);
    otherwise columns of one size share launches, and ``graph`` captures the
    whole commit once per buffer set and replays it."""

    def __init__(self, log_sizes, log_blowup: int, tree: TwiddleTree, m31: bool = False, per_column: bool = False,
                 graph: bool = False, stream=None):
        ffi.init()
        self.stream = as_stream(stream)
        self._tree = tree  # the library keeps its device pointers: keep the buffers alive
        self.log_sizes = [int(x) for x in log_sizes]
        flags = (1 if per_column else 0) | (2 if graph else 0)
        h = C.c_void_p()
        ffi.call("stwo_b200_committer_create", _u32_array(self.log_sizes), C.c_uint32(len(self.log_sizes)),
                 C.c_uint32(log_blowup), C.c_int(1 if m31 else 0), C.c_void_p(tree.twiddles.ptr),
                 C.c_void_p(tree.itwiddles.ptr), C.c_uint32(tree.log_size), C.c_uint32(flags), C.byref(h))
        self._h = h
        L = C.c_uint32(0)
        ffi.call("stwo_b200_committer_lifting_log_size", h, C.byref(L))
        self.lifting_log_size = L.value

    def new_layers(self):
        return [DeviceBuffer(32 << k, self.stream) for k in range(self.lifting_log_size + 1)]

    def commit(self, evals, coeffs, ldes, layers):
        ffi.call("stwo_b200_committer_commit", self._h, _ptr_array(evals), _ptr_array(coeffs), _ptr_array(ldes),
                 _ptr_array(layers), self.stream)
        return layers

    def commit_from_host(self, host_ptrs, evals, coeffs, ldes, layers):
        """commit() with the columns in host memory: ``host_ptrs[i]`` is the
        address of column i (pinned for asynchronous copies), copied into
        ``evals[i]`` one size group at a time while the groups already on the
        device are transformed."""
        if len(host_ptrs) != len(self.log_sizes):
            raise ValueError("one host column per committed column")
        hp = (C.c_void_p * len(host_ptrs))(*[C.c_void_p(int(p)) for p in host_ptrs])
        ffi.call("stwo_b200_committer_commit_from_host", self._h, hp, _ptr_array(evals), _ptr_array(coeffs),
                 _ptr_array(ldes), _ptr_array(layers), self.stream)
        return layers

    def autotune(self, evals, coeffs, ldes, cache_path: str | None = None, reps: int = 3):
        path = cache_path.encode() if cache_path else None
        ffi.call("stwo_b200_committer_autotune", self._h, _ptr_array(evals), _ptr_array(coeffs), _ptr_array(ldes),
                 C.c_char_p(path), C.c_uint32(reps))

    def close(self):
        if self._h:
            ffi.call("stwo_b200_committer_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
