"""ORACLE — test infrastructure only.

ctypes bindings of ``liboracle.so``, the CPU restatement of stwo's SimdBackend
for the commit + FRI path.  Used by ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline legs of ``bench.py`` as the checker; never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

P = (1 << 31) - 1
_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

U32P = C.POINTER(C.c_uint32)
U8P = C.POINTER(C.c_uint8)


def build() -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _lib.oracle_last_error.restype = C.c_char_p
        _lib.oracle_channel_grind.restype = C.c_uint64
        _lib.oracle_last_intermediate.restype = C.c_size_t
    return _lib


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def _p(a: np.ndarray):
    return a.ctypes.data_as(U32P)


def _p8(a: np.ndarray):
    return a.ctypes.data_as(U8P)


def _ptrs(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().oracle_last_error().decode())


def set_threads(n: int) -> int:
    return lib().oracle_set_threads(C.c_int(n))


def blake2s(data: bytes, m31: bool = False) -> bytes:
    out = (C.c_uint8 * 32)()
    buf = (C.c_uint8 * max(1, len(data))).from_buffer_copy(data or b"\0")
    lib().oracle_blake2s(buf, C.c_size_t(len(data)), C.c_int(int(m31)), out)
    return bytes(out)


def index_to_point(index: int):
    xy = (C.c_uint32 * 2)()
    lib().oracle_index_to_point(C.c_uint64(index), xy)
    return int(xy[0]), int(xy[1])


def qm31_mul(a, b) -> tuple:
    x, y, out = _u32(a), _u32(b), np.zeros(4, np.uint32)
    _check(lib().oracle_qm31_mul(_p(x), _p(y), _p(out)))
    return tuple(int(v) for v in out)


def qm31_inv(a) -> tuple:
    x, out = _u32(a), np.zeros(4, np.uint32)
    _check(lib().oracle_qm31_inv(_p(x), _p(out)))
    return tuple(int(v) for v in out)


def canonic_half_initial_index(log_size: int) -> int:
    """CanonicCoset(log_size).circle_domain().half_coset initial index."""
    return 1 << (31 - (log_size + 1))


def canonic_half_coset_root(log_size: int):
    """(initial_index, log_size) of CanonicCoset(log_size).half_coset."""
    return canonic_half_initial_index(log_size), log_size - 1


def bit_reverse(v) -> np.ndarray:
    a = _u32(v).copy()
    lib().oracle_bit_reverse(_p(a), C.c_uint32(int(a.size).bit_length() - 1))
    return a


def precompute_twiddles(initial_index: int, log_size: int):
    n = 1 << log_size
    tw = np.zeros(n, np.uint32)
    itw = np.zeros(n, np.uint32)
    _check(lib().oracle_precompute_twiddles(C.c_uint64(initial_index), C.c_uint32(log_size), _p(tw), _p(itw)))
    return tw, itw


def interpolate(values, itw, half_initial_index=None) -> np.ndarray:
    a = _u32(values).copy()
    log_n = int(a.size).bit_length() - 1
    if half_initial_index is None:
        half_initial_index = canonic_half_initial_index(log_n)
    itw = _u32(itw)
    _check(lib().oracle_interpolate(_p(a), C.c_uint32(log_n), C.c_uint64(half_initial_index), _p(itw),
                                    C.c_size_t(itw.size)))
    return a


def interpolate_columns(cols, itw):
    arrs = [_u32(c).copy() for c in cols]
    logs = _u32([int(a.size).bit_length() - 1 for a in arrs])
    itw = _u32(itw)
    _check(lib().oracle_interpolate_columns(_ptrs(arrs), _p(logs), C.c_uint32(len(arrs)), _p(itw),
                                            C.c_size_t(itw.size)))
    return arrs


def evaluate(coeffs, log_eval: int, tw, half_initial_index=None) -> np.ndarray:
    c = _u32(coeffs)
    log_n = int(c.size).bit_length() - 1
    if half_initial_index is None:
        half_initial_index = canonic_half_initial_index(log_eval)
    out = np.zeros(1 << log_eval, np.uint32)
    tw = _u32(tw)
    _check(lib().oracle_evaluate(_p(c), C.c_uint32(log_n), C.c_uint32(log_eval), C.c_uint64(half_initial_index),
                                 _p(tw), C.c_size_t(tw.size), _p(out)))
    return out


def evaluate_columns(coeffs, log_blowup: int, tw):
    arrs = [_u32(c) for c in coeffs]
    logs = _u32([int(a.size).bit_length() - 1 for a in arrs])
    outs = [np.zeros(a.size << log_blowup, np.uint32) for a in arrs]
    tw = _u32(tw)
    _check(lib().oracle_evaluate_columns(_ptrs(arrs), _p(logs), C.c_uint32(len(arrs)), C.c_uint32(log_blowup),
                                         _p(tw), C.c_size_t(tw.size), _ptrs(outs)))
    return outs


def eval_at_point_m31(coeffs, x: int, y: int) -> int:
    c = _u32(coeffs)
    out = C.c_uint32()
    _check(lib().oracle_eval_at_point_m31(_p(c), C.c_uint32(int(c.size).bit_length() - 1), C.c_uint32(x),
                                          C.c_uint32(y), C.byref(out)))
    return int(out.value)


def merkle_build_layers(cols, lifting_log_size: int, m31: bool = False, staged: bool = False):
    """Lifted Merkle layers, root first; each layer a (2^k, 32) uint8 array.
    staged: the leaves in SimdBackend's staged form (the same hashes, fewer
    compressions for columns of different sizes)."""
    arrs = [_u32(c) for c in cols]
    logs = _u32([int(a.size).bit_length() - 1 for a in arrs])
    L = lifting_log_size
    out = np.zeros(((1 << (L + 1)) - 1) * 32, np.uint8)
    _check(lib().oracle_merkle_build_layers(_ptrs(arrs) if arrs else None, _p(logs), C.c_uint32(len(arrs)),
                                            C.c_uint32(L), C.c_int(int(m31)), C.c_int(int(staged)), _p8(out)))
    layers, off = [], 0
    for k in range(L + 1):
        layers.append(out[off * 32:(off + (1 << k)) * 32].reshape(1 << k, 32))
        off += 1 << k
    return layers


def merkle_build_leaves(cols, lifting_log_size: int, m31: bool = False) -> np.ndarray:
    arrs = [_u32(c) for c in cols]
    logs = _u32([int(a.size).bit_length() - 1 for a in arrs])
    n = 1 << lifting_log_size if arrs else 1
    out = np.zeros(n * 32, np.uint8)
    _check(lib().oracle_merkle_build_leaves(_ptrs(arrs) if arrs else None, _p(logs), C.c_uint32(len(arrs)),
                                            C.c_uint32(lifting_log_size), C.c_int(int(m31)), _p8(out)))
    return out.reshape(n, 32)


def merkle_next_layer(prev: np.ndarray, m31: bool = False) -> np.ndarray:
    prev = np.ascontiguousarray(prev, np.uint8).reshape(-1, 32)
    lp = prev.shape[0].bit_length() - 1
    out = np.zeros((prev.shape[0] // 2) * 32, np.uint8)
    _check(lib().oracle_merkle_next_layer(_p8(prev), C.c_uint32(lp), C.c_int(int(m31)), _p8(out)))
    return out.reshape(-1, 32)


def commit_on_layer(log_size: int, prev, cols, m31: bool = False) -> np.ndarray:
    arrs = [_u32(c) for c in cols]
    pv = None if prev is None else np.ascontiguousarray(prev, np.uint8).reshape(-1)
    out = np.zeros((1 << log_size) * 32, np.uint8)
    _check(lib().oracle_commit_on_layer(C.c_uint32(log_size), None if pv is None else _p8(pv),
                                        _ptrs(arrs) if arrs else None, C.c_uint32(len(arrs)), C.c_int(int(m31)),
                                        _p8(out)))
    return out.reshape(-1, 32)


def mixed_degree_commit(cols, m31: bool = False):
    """MerkleProver::commit (prover/vcs/prover.rs:39-65): layers root first."""
    if not cols:
        return [commit_on_layer(0, None, [], m31)]
    order = sorted(range(len(cols)), key=lambda i: -len(cols[i]))
    cols = [cols[i] for i in order]
    max_log = len(cols[0]).bit_length() - 1
    layers, pos = [], 0
    for log_size in range(max_log, -1, -1):
        layer_cols = []
        while pos < len(cols) and len(cols[pos]).bit_length() - 1 == log_size:
            layer_cols.append(cols[pos])
            pos += 1
        layers.append(commit_on_layer(log_size, layers[-1] if layers else None, layer_cols, m31))
    return layers[::-1]


def _alpha(alpha):
    return _u32(alpha)


def fold_line(cols4, itw, alpha, fold_step: int = 1):
    ins = [_u32(c) for c in cols4]
    log_m = int(ins[0].size).bit_length() - 1
    outs = [np.zeros(ins[0].size >> fold_step, np.uint32) for _ in range(4)]
    itw = _u32(itw)
    a = _alpha(alpha)
    _check(lib().oracle_fold_line(_ptrs(ins), C.c_uint32(log_m), _p(itw), C.c_size_t(itw.size), _p(a),
                                  C.c_uint32(fold_step), _ptrs(outs)))
    return outs


def fold_line_direct(cols4, initial_index: int, alpha):
    ins = [_u32(c) for c in cols4]
    log_m = int(ins[0].size).bit_length() - 1
    outs = [np.zeros(ins[0].size >> 1, np.uint32) for _ in range(4)]
    a = _alpha(alpha)
    _check(lib().oracle_fold_line_direct(_ptrs(ins), C.c_uint64(initial_index), C.c_uint32(log_m), _p(a),
                                         _ptrs(outs)))
    return outs


def fold_circle_into_line(dst4, src4, itw, alpha, half_initial_index=None):
    dst = [_u32(c).copy() for c in dst4]
    src = [_u32(c) for c in src4]
    log_n = int(src[0].size).bit_length() - 1
    if half_initial_index is None:
        half_initial_index = canonic_half_initial_index(log_n)
    itw = _u32(itw)
    a = _alpha(alpha)
    _check(lib().oracle_fold_circle_into_line(_ptrs(dst), _ptrs(src), C.c_uint64(half_initial_index),
                                              C.c_uint32(log_n), _p(itw), C.c_size_t(itw.size), _p(a)))
    return dst


def fold_circle_into_line_direct(dst4, src4, half_initial_index: int, alpha):
    dst = [_u32(c).copy() for c in dst4]
    src = [_u32(c) for c in src4]
    log_n = int(src[0].size).bit_length() - 1
    a = _alpha(alpha)
    _check(lib().oracle_fold_circle_into_line_direct(_ptrs(dst), _ptrs(src), C.c_uint64(half_initial_index),
                                                     C.c_uint32(log_n), _p(a)))
    return dst


def decompose(cols4):
    ins = [_u32(c) for c in cols4]
    log_n = int(ins[0].size).bit_length() - 1
    outs = [np.zeros_like(ins[0]) for _ in range(4)]
    lam = np.zeros(4, np.uint32)
    _check(lib().oracle_decompose(_ptrs(ins), C.c_uint32(log_n), _ptrs(outs), _p(lam)))
    return outs, lam


# ---- QuotientOps / AccumulationOps / eval_at_point (oracle_pcs.cpp) ----
def accumulate_numerators(cols, log_n: int, point, terms):
    """One sample batch: terms = [(column index, value (4 words), alpha (4
    words)), ...]; returns (4 partial-numerator columns, first linear term)."""
    arrs = [_u32(c) for c in cols]
    idx = _u32([t[0] for t in terms])
    vals = _u32(np.asarray([t[1] for t in terms], np.uint32).reshape(-1))
    alps = _u32(np.asarray([t[2] for t in terms], np.uint32).reshape(-1))
    outs = [np.zeros(1 << log_n, np.uint32) for _ in range(4)]
    first = np.zeros(4, np.uint32)
    pt = _u32(np.asarray(point, np.uint32).reshape(-1))
    rc = lib().oracle_accumulate_numerators(_ptrs(arrs), C.c_uint32(len(arrs)), C.c_uint32(log_n), _p(pt), _p(idx),
                                            _p(vals), _p(alps), C.c_uint32(len(terms)), _ptrs(outs), _p(first))
    if rc != 0:
        raise RuntimeError("oracle: accumulate_numerators failed")
    return outs, first


def compute_quotients_and_combine(accs, lifting_log: int):
    """accs = [(point (8 words), 4 partial columns, first linear term (4)), ...]."""
    pts = _u32(np.asarray([a[0] for a in accs], np.uint32).reshape(-1))
    parts = [_u32(c) for a in accs for c in a[1]]
    logs = _u32([int(a[1][0].size).bit_length() - 1 for a in accs])
    firsts = _u32(np.asarray([a[2] for a in accs], np.uint32).reshape(-1))
    outs = [np.zeros(1 << lifting_log, np.uint32) for _ in range(4)]
    rc = lib().oracle_compute_quotients_and_combine(_p(pts), _ptrs(parts), _p(logs), _p(firsts),
                                                    C.c_uint32(len(accs)), C.c_uint32(lifting_log), _ptrs(outs))
    if rc != 0:
        raise RuntimeError("oracle: compute_quotients_and_combine failed")
    return outs


def lift_and_accumulate(cols4_list):
    """cols4_list: secure columns (4 coordinate arrays each), strictly increasing sizes."""
    arrs = [_u32(c) for cols4 in cols4_list for c in cols4]
    logs = _u32([int(c4[0].size).bit_length() - 1 for c4 in cols4_list])
    outs = [np.zeros(cols4_list[-1][0].size, np.uint32) for _ in range(4)]
    if lib().oracle_lift_and_accumulate(_ptrs(arrs), _p(logs), C.c_uint32(len(cols4_list)), _ptrs(outs)) != 0:
        raise RuntimeError("oracle: lift_and_accumulate failed")
    return outs


def accumulate(col4, other4):
    out = [np.array(c, dtype=np.uint32) for c in col4]
    oth = [_u32(c) for c in other4]
    lib().oracle_accumulate(_ptrs(out), _ptrs(oth), C.c_size_t(out[0].size))
    return out


def generate_secure_powers(felt, n: int) -> np.ndarray:
    f = _u32(np.asarray(felt, np.uint32).reshape(-1))
    out = np.zeros(4 * n, np.uint32)
    lib().oracle_generate_secure_powers(_p(f), C.c_uint32(n), _p(out))
    return out.reshape(n, 4)


def eval_at_secure_point(coeffs, point) -> np.ndarray:
    c = _u32(coeffs)
    pt = _u32(np.asarray(point, np.uint32).reshape(-1))
    out = np.zeros(4, np.uint32)
    lib().oracle_eval_at_secure_point(_p(c), C.c_uint32(int(c.size).bit_length() - 1), _p(pt), _p(out))
    return out


class ChannelState(C.Structure):
    _fields_ = [("digest", C.c_uint8 * 32), ("n_draws", C.c_uint32), ("m31", C.c_int32)]


class Channel:
    """Blake2s Fiat-Shamir channel (core/channel/blake2s.rs)."""

    def __init__(self, m31: bool = False):
        self.s = ChannelState()
        self.s.m31 = int(m31)

    @property
    def digest(self) -> bytes:
        return bytes(self.s.digest)

    @property
    def n_draws(self) -> int:
        return int(self.s.n_draws)

    def mix_u32s(self, words):
        w = _u32(words)
        lib().oracle_channel_mix_u32s(C.byref(self.s), _p(w), C.c_size_t(w.size))

    def mix_u64(self, v: int):
        lib().oracle_channel_mix_u64(C.byref(self.s), C.c_uint64(v))

    def mix_felts(self, felts):
        f = _u32(np.asarray(felts, dtype=np.uint32).reshape(-1))
        lib().oracle_channel_mix_felts(C.byref(self.s), _p(f), C.c_size_t(f.size // 4))

    def mix_root(self, root: bytes):
        r = (C.c_uint8 * 32).from_buffer_copy(bytes(root))
        lib().oracle_channel_mix_root(C.byref(self.s), r)

    def draw_u32s(self):
        out = np.zeros(8, np.uint32)
        lib().oracle_channel_draw_u32s(C.byref(self.s), _p(out))
        return out

    def draw_secure_felts(self, n: int):
        out = np.zeros(4 * n, np.uint32)
        lib().oracle_channel_draw_secure_felts(C.byref(self.s), C.c_size_t(n), _p(out))
        return out.reshape(n, 4)

    def draw_secure_felt(self):
        return self.draw_secure_felts(1)[0]

    def verify_pow(self, bits: int, nonce: int) -> bool:
        return bool(lib().oracle_channel_verify_pow(C.byref(self.s), C.c_uint32(bits), C.c_uint64(nonce)))

    def grind(self, bits: int) -> int:
        return int(lib().oracle_channel_grind(C.byref(self.s), C.c_uint32(bits)))


class WideFibConfig(C.Structure):
    _fields_ = [("log_n_rows", C.c_uint32), ("n_cols", C.c_uint32), ("log_blowup", C.c_uint32),
                ("pow_bits", C.c_uint32), ("n_queries", C.c_uint32), ("log_last_layer_degree_bound", C.c_uint32),
                ("line_fold_step", C.c_uint32), ("m31_channel", C.c_int32)]


def wide_fib_config(log_n_rows: int, n_cols: int = 100, log_blowup: int = 1, pow_bits: int = 10, n_queries: int = 3,
                    log_last_layer_degree_bound: int = 0, line_fold_step: int = 1, m31_channel: bool = False):
    return WideFibConfig(log_n_rows, n_cols, log_blowup, pow_bits, n_queries, log_last_layer_degree_bound,
                         line_fold_step, int(m31_channel))


def wide_fib_inputs(log_n_rows: int, seed: int):
    """First two trace columns, uniform in [0, P) (seeded numpy PCG64)."""
    r = np.random.default_rng(seed)
    return (r.integers(0, P, 1 << log_n_rows, dtype=np.uint32), r.integers(0, P, 1 << log_n_rows, dtype=np.uint32))


def prove_wide_fib(cfg: WideFibConfig, a, b) -> bytes:
    a, b = _u32(a), _u32(b)
    n = C.c_size_t()
    _check(lib().oracle_prove_wide_fib(C.byref(cfg), _p(a), _p(b), C.byref(n)))
    out = (C.c_uint8 * n.value)()
    lib().oracle_last_proof(out)
    return bytes(out)


def fri_inputs(log_n: int, seed: int, n_queries: int = 70):
    """Seeded FRI-heavy inputs: 4 coordinate columns uniform in [0, P), one QM31
    folding alpha per fold (log_n of them, as a (log_n, 4) array), and the
    sorted distinct query positions drawn from n_queries uniform draws."""
    r = np.random.default_rng(seed)
    n = 1 << log_n
    coords = [r.integers(0, P, n, dtype=np.uint32) for _ in range(4)]
    alphas = r.integers(0, P, (log_n, 4), dtype=np.uint32)
    queries = np.unique(r.integers(0, n, n_queries, dtype=np.uint64))
    return coords, alphas, queries


def fri_prove_seeded(coords, log_n: int, alphas, queries, m31: bool = False) -> bytes:
    """FriProver commit + decommit of one secure column with the given alphas
    (FriProof bytes: first layer, inner layers, last-layer value)."""
    arrs = [_u32(c) for c in coords]
    a = np.ascontiguousarray(alphas, dtype=np.uint32).reshape(-1)
    q = np.ascontiguousarray(queries, dtype=np.uint64)
    n = C.c_size_t()
    _check(lib().oracle_fri_prove_seeded(_ptrs(arrs), C.c_uint32(log_n), _p(a),
                                         q.ctypes.data_as(C.POINTER(C.c_uint64)), C.c_size_t(q.size),
                                         C.c_int(1 if m31 else 0), C.byref(n)))
    out = (C.c_uint8 * n.value)()
    lib().oracle_last_proof(out)
    return bytes(out)


def last_intermediate(which: int, k: int) -> np.ndarray:
    n = lib().oracle_last_intermediate(C.c_int(which), C.c_int(k), None)
    out = np.zeros(n, np.uint32)
    lib().oracle_last_intermediate(C.c_int(which), C.c_int(k), _p(out))
    return out


def last_roots(n_trees: int = 3):
    out = (C.c_uint8 * (32 * n_trees))()
    lib().oracle_last_roots(out)
    return [bytes(out[32 * i:32 * (i + 1)]) for i in range(n_trees)]


def verify_wide_fib(proof: bytes, log_n_rows: int, n_cols: int, m31: bool = False):
    """Returns None when the proof verifies, else the rejection reason."""
    buf = (C.c_uint8 * len(proof)).from_buffer_copy(proof)
    rc = lib().oracle_verify_wide_fib(buf, C.c_size_t(len(proof)), C.c_uint32(log_n_rows), C.c_uint32(n_cols),
                                      C.c_int(int(m31)))
    return None if rc == 0 else lib().oracle_last_error().decode()
