"""Pins the CPU oracle (stwo SimdBackend restatement) to the reference's own
known-answer tests and structural identities.  No GPU needed."""
import hashlib

import numpy as np
import pytest

P = (1 << 31) - 1


def test_blake2s_kat(oracle):
    # core/vcs/blake2_hash.rs:134-139
    assert oracle.blake2s(b"a").hex() == "4a0d129873403037c2cd9b9048203687f6233fb6738956e0349bd4320fec3e90"
    # core/vcs/blake2_hash.rs:142-152: streaming == one-shot; empty input
    assert oracle.blake2s(b"ab") == hashlib.blake2s(b"ab").digest()
    assert oracle.blake2s(b"") == hashlib.blake2s(b"").digest()


@pytest.mark.parametrize("n", [0, 1, 63, 64, 65, 127, 128, 129, 1000])
def test_blake2s_vs_hashlib(oracle, n):
    data = bytes((i * 7 + 3) & 0xFF for i in range(n))
    assert oracle.blake2s(data) == hashlib.blake2s(data).digest()


def test_blake2s_m31_output(oracle):
    # core/vcs/blake2_hash.rs:110-118: every LE word reduced mod P
    h = hashlib.blake2s(b"xyz").digest()
    words = np.frombuffer(h, np.uint32).astype(np.uint64)
    red = ((((words >> 31) + words + 1) >> 31) + words) & P
    assert oracle.blake2s(b"xyz", m31=True) == red.astype(np.uint32).tobytes()


def test_channel_mix_u64_kat(oracle):
    # core/channel/blake2s.rs:213-232
    c = oracle.Channel()
    c.mix_u64(0x1111222233334444)
    d = c.digest
    c2 = oracle.Channel()
    c2.mix_u32s([0x33334444, 0x11112222])
    assert d == c2.digest
    assert d == bytes([0xbc, 0x9e, 0x3f, 0xc1, 0xd2, 0x4e, 0x88, 0x97, 0x95, 0x6d, 0x33, 0x59, 0x32, 0x73,
                       0x97, 0x24, 0x9d, 0x6b, 0xca, 0xcd, 0x22, 0x4d, 0x92, 0x74, 0x4, 0xe7, 0xba, 0x4a,
                       0x77, 0xdc, 0x6e, 0xce])


def test_channel_mix_u32s_kat(oracle):
    # core/channel/blake2s.rs:234-247
    c = oracle.Channel()
    c.mix_u32s([1, 2, 3, 4, 5, 6, 7, 8, 9])
    assert c.digest == bytes([0x70, 0x91, 0x76, 0x83, 0x57, 0xbb, 0x1b, 0xb3, 0x34, 0x6f, 0xda, 0xb6, 0xb3, 0x57,
                              0xd7, 0xfa, 0x46, 0xb8, 0xfb, 0xe3, 0x2c, 0x2e, 0x43, 0x24, 0xa0, 0xff, 0xc2, 0x94,
                              0xcb, 0xf9, 0xa1, 0xc7])


def test_channel_draw_counts(oracle):
    # core/channel/blake2s.rs:153-164
    c = oracle.Channel()
    c.draw_u32s()
    assert c.n_draws == 1
    c.draw_secure_felts(9)
    assert c.n_draws == 6


def test_channel_draw_definition(oracle):
    # draw_u32s = Blake2s(digest || LE32(n_draws) || 0x00)
    c = oracle.Channel()
    c.mix_u32s([5])
    d = c.digest
    w = c.draw_u32s()
    assert w.tobytes() == hashlib.blake2s(d + (0).to_bytes(4, "little") + b"\0").digest()


def test_pow_prefix_and_grind(oracle):
    # core/channel/blake2s.rs:122-140, prover/backend/simd/grind.rs:25-60
    c = oracle.Channel()
    c.mix_u64(42)
    nonce = c.grind(8)
    assert c.verify_pow(8, nonce)
    pre = hashlib.blake2s((0x12345678).to_bytes(4, "little") + bytes(12) + c.digest +
                          (8).to_bytes(4, "little")).digest()
    for k in range(nonce):
        h = hashlib.blake2s(pre + k.to_bytes(8, "little")).digest()
        assert int.from_bytes(h[:4], "little") & 0xFF != 0
    h = hashlib.blake2s(pre + nonce.to_bytes(8, "little")).digest()
    assert int.from_bytes(h[:4], "little") & 0xFF == 0


def test_domain_line_twiddles_slicing(oracle):
    # core/poly/utils.rs:141-148: CanonicCoset(4).circle_domain() line domain
    # over buffer [0..8) -> layers [0,1,2,3], [4,5], [6].
    buf = np.arange(8, dtype=np.uint32)
    line_log = 3
    layers = [buf[8 - (1 << (line_log - i)): 8 - (1 << (line_log - i - 1))] for i in range(line_log)]
    assert [list(x) for x in layers] == [[0, 1, 2, 3], [4, 5], [6]]


def test_twiddles_are_coset_x_bitreversed(oracle):
    # prover/backend/cpu/circle.rs:294-311
    init, log = oracle.canonic_half_coset_root(6)
    tw, itw = oracle.precompute_twiddles(init, log)
    assert tw.size == 1 << log and tw[-1] == 1
    step = 1 << (31 - log)
    first = [oracle.index_to_point((init + step * j) % (1 << 31))[0] for j in range(1 << (log - 1))]
    assert list(tw[:1 << (log - 1)]) == list(oracle.bit_reverse(np.array(first, np.uint32)))
    prod = (tw.astype(np.uint64) * itw.astype(np.uint64)) % P
    assert (prod == 1).all()


def _domain_point(oracle, log_size, j):
    """Canonic circle domain point at bit-reversed position j."""
    jj = int(format(j, f"0{log_size}b")[::-1], 2)
    half_init = oracle.canonic_half_initial_index(log_size)
    hs = 1 << (log_size - 1)
    step = 1 << (31 - (log_size - 1))
    if jj < hs:
        idx = (half_init + step * jj) % (1 << 31)
    else:
        idx = ((1 << 31) - (half_init + step * (jj - hs)) % (1 << 31)) % (1 << 31)
    return oracle.index_to_point(idx)


@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("log_blowup", [0, 1, 2])
def test_fft_vs_naive_evaluation(oracle, log_n, log_blowup):
    # prover/backend/simd/fft/rfft.rs:717-746, ifft.rs:687-718 (ground truth)
    rng = np.random.default_rng(100 * log_n + log_blowup)
    tw, itw = oracle.precompute_twiddles(*oracle.canonic_half_coset_root(log_n + 3))
    coeffs = rng.integers(0, P, 1 << log_n, dtype=np.uint32)
    le = log_n + log_blowup
    ev = oracle.evaluate(coeffs, le, tw)
    for j in range(1 << le):
        x, y = _domain_point(oracle, le, j)
        assert oracle.eval_at_point_m31(coeffs, x, y) == ev[j]
    if log_blowup == 0:
        assert (oracle.interpolate(ev, itw) == coeffs).all()


@pytest.mark.parametrize("log_n", [8, 12, 16, 17])
def test_fft_roundtrip(oracle, log_n):
    rng = np.random.default_rng(log_n)
    tw, itw = oracle.precompute_twiddles(*oracle.canonic_half_coset_root(log_n + 1))
    vals = rng.integers(0, P, 1 << log_n, dtype=np.uint32)
    coeffs = oracle.interpolate(vals, itw)
    assert (oracle.evaluate(coeffs, log_n, tw) == vals).all()
    ext = oracle.evaluate(coeffs, log_n + 1, tw)
    # the extension restricted back interpolates to the zero-padded polynomial
    back = oracle.interpolate(ext, itw)
    assert (back[:1 << log_n] == coeffs).all() and (back[1 << log_n:] == 0).all()


def test_lifted_leaf_layouts(oracle):
    # prover/vcs_lifted/prover.rs:228-275
    cols = [np.arange(1 << i, dtype=np.uint32) for i in range(2, 5)]
    layers = oracle.merkle_build_layers(cols, 4)
    leaves = layers[-1]
    assert bytes(leaves[0]) == hashlib.blake2s(bytes(12)).digest()
    le = lambda *w: b"".join(int(x).to_bytes(4, "little") for x in w)
    assert bytes(leaves[4]) == hashlib.blake2s(le(0, 2, 4)).digest()
    assert bytes(leaves[15]) == hashlib.blake2s(le(3, 7, 15)).digest()
    # layers root-first, parent = H(left || right)
    for k in range(4):
        for i in range(1 << k):
            assert bytes(layers[k][i]) == hashlib.blake2s(bytes(layers[k + 1][2 * i]) +
                                                          bytes(layers[k + 1][2 * i + 1])).digest()


def test_lifted_leaves_streaming_definition(oracle):
    # cpu/merkle_lifted.rs:44-78: per-leaf byte stream over columns sorted by
    # length (stable), lifted index ((i >> (r+1)) << 1) + (i & 1).
    rng = np.random.default_rng(7)
    logs = [5, 3, 5, 1, 4, 3] + [4] * 17
    cols = [rng.integers(0, P, 1 << l, dtype=np.uint32) for l in logs]
    L = 6
    layers = oracle.merkle_build_layers(cols, L)
    order = sorted(range(len(cols)), key=lambda i: logs[i])
    for i in [0, 1, 2, 3, 17, 40, 63]:
        data = b""
        for c in order:
            r = L - logs[c]
            idx = i if r == 0 else ((i >> (r + 1)) << 1) + (i & 1)
            data += int(cols[c][idx]).to_bytes(4, "little")
        assert bytes(layers[-1][i]) == hashlib.blake2s(data).digest()


@pytest.mark.parametrize("logs,L,m31", [
    ([5, 3, 5, 1, 4, 3] + [4] * 17, 6, False),
    ([2] * 16 + [3] * 16, 3, True),                       # whole blocks, the last at L
    ([1] * 5 + [2] * 40 + [6] * 3 + [7] * 20, 9, False),  # last block alone at L > max
    ([4], 4, True),
])
def test_lifted_leaves_staged_form(oracle, logs, L, m31):
    # simd/blake2s_lifted.rs:42-160: message blocks hashed at the size of
    # their largest column, chaining values lifted block to block; the same
    # leaves as the per-leaf byte stream of cpu/merkle_lifted.rs:44-78.
    rng = np.random.default_rng(len(logs) + L)
    cols = [rng.integers(0, P, 1 << l, dtype=np.uint32) for l in logs]
    direct = oracle.merkle_build_layers(cols, L, m31)
    staged = oracle.merkle_build_layers(cols, L, m31, staged=True)
    for k in range(L + 1):
        assert (direct[k] == staged[k]).all(), k


def test_lifted_equals_mixed_degree_on_lifted_input(oracle):
    # prover/vcs_lifted/prover.rs:307-336
    LOG, LIFT = 3, 9
    tw, itw = oracle.precompute_twiddles(*oracle.canonic_half_coset_root(LIFT))
    coeffs = np.arange(1 << LOG, dtype=np.uint32)
    lifted_coeffs = np.zeros(1 << LIFT, np.uint32)
    # lift_poly: evaluations of p(pi^(LIFT-LOG)(.)) -- computed via the lifted
    # leaf index map on the small evaluation.
    small = oracle.evaluate(coeffs, LOG, tw)
    r = LIFT - LOG
    lifted_eval = np.array([small[((i >> (r + 1)) << 1) + (i & 1)] for i in range(1 << LIFT)], np.uint32)
    zero = np.zeros(1 << LIFT, np.uint32)
    mixed = oracle.mixed_degree_commit([lifted_eval, zero])
    lifted1 = oracle.merkle_build_layers([lifted_eval, zero], LIFT)
    lifted2 = oracle.merkle_build_layers([small, zero], LIFT)
    assert bytes(lifted1[0][0]) == bytes(lifted2[0][0]) == bytes(mixed[0][0])
    del lifted_coeffs


def test_empty_columns_commit(oracle):
    # prover/vcs_lifted/prover.rs:216-228
    lifted = oracle.merkle_build_layers([], 0)
    mixed = oracle.mixed_degree_commit([])
    assert bytes(lifted[0][0]) == bytes(mixed[0][0]) == hashlib.blake2s(b"").digest()


def test_fold_line_tree_equals_direct(oracle):
    # cpu/fri.rs:67-92 vs simd/fri.rs:32-122 (twiddle-tree x^-1)
    rng = np.random.default_rng(3)
    for log_m in [1, 2, 5, 8]:
        root_log = log_m + 2
        init, lg = oracle.canonic_half_coset_root(root_log)
        tw, itw = oracle.precompute_twiddles(init, lg)
        # line domain = CanonicCoset(log_m + 1).half_coset = half_odds(log_m)
        dom_init = oracle.canonic_half_initial_index(log_m + 1)
        cols = [rng.integers(0, P, 1 << log_m, dtype=np.uint32) for _ in range(4)]
        alpha = rng.integers(0, P, 4, dtype=np.uint32)
        a = oracle.fold_line(cols, itw, alpha, 1)
        b = oracle.fold_line_direct(cols, dom_init, alpha)
        for k in range(4):
            assert (a[k] == b[k]).all()


def test_fold_circle_tree_equals_direct(oracle):
    rng = np.random.default_rng(4)
    for log_n in [2, 3, 6, 9]:
        init, lg = oracle.canonic_half_coset_root(log_n + 1)
        tw, itw = oracle.precompute_twiddles(init, lg)
        src = [rng.integers(0, P, 1 << log_n, dtype=np.uint32) for _ in range(4)]
        dst = [rng.integers(0, P, 1 << (log_n - 1), dtype=np.uint32) for _ in range(4)]
        alpha = rng.integers(0, P, 4, dtype=np.uint32)
        a = oracle.fold_circle_into_line(dst, src, itw, alpha)
        b = oracle.fold_circle_into_line_direct(dst, src, oracle.canonic_half_initial_index(log_n), alpha)
        for k in range(4):
            assert (a[k] == b[k]).all()


def test_fold_of_low_degree_is_low_degree(oracle):
    # FRI soundness identity: folding evaluations of a degree < 2^k poly on a
    # blowup-2 domain gives a degree < 2^(k-1) line evaluation, which the
    # next fold sends to a constant after enough steps.
    log_n = 6
    init, lg = oracle.canonic_half_coset_root(log_n)
    tw, itw = oracle.precompute_twiddles(init, lg)
    rng = np.random.default_rng(9)
    coords = []
    for _ in range(4):
        c = np.zeros(1 << log_n, np.uint32)
        c[:1 << (log_n - 1)] = rng.integers(0, P, 1 << (log_n - 1), dtype=np.uint32)
        coords.append(oracle.evaluate(c[:1 << (log_n - 1)], log_n, tw))
    alpha = rng.integers(0, P, 4, dtype=np.uint32)
    dst = [np.zeros(1 << (log_n - 1), np.uint32) for _ in range(4)]
    line = oracle.fold_circle_into_line(dst, coords, itw, alpha)
    cur = line
    for _ in range(log_n - 2):
        cur = oracle.fold_line(cur, itw, alpha, 1)
    # blowup 2 -> after log_n-2 line folds a line evaluation of size 2 of a
    # constant: both entries equal.
    for k in range(4):
        assert cur[k][0] == cur[k][1]


def test_decompose_small_lambda_zero(oracle):
    rng = np.random.default_rng(5)
    cols = [rng.integers(0, P, 8, dtype=np.uint32) for _ in range(4)]
    g, lam = oracle.decompose(cols)
    assert (lam == 0).all()
    for k in range(4):
        assert (g[k] == cols[k]).all()


@pytest.mark.parametrize("log_n,cols,m31", [(4, 100, False), (5, 8, True), (8, 100, False), (6, 3, False),
                                            (10, 16, False)])
def test_wide_fib_prove_verify(oracle, log_n, cols, m31):
    # examples/src/wide_fibonacci/mod.rs:188-244: prove then verify; tampered
    # proofs are rejected.
    a, b = oracle.wide_fib_inputs(log_n, 7)
    cfg = oracle.wide_fib_config(log_n, cols, m31_channel=m31)
    proof = oracle.prove_wide_fib(cfg, a, b)
    assert oracle.verify_wide_fib(proof, log_n, cols, m31) is None
    assert oracle.prove_wide_fib(cfg, a, b) == proof  # deterministic
    rng = np.random.default_rng(log_n)
    for pos in rng.integers(8, len(proof), 12):
        bad = bytearray(proof)
        bad[int(pos)] ^= 0x10
        assert oracle.verify_wide_fib(bytes(bad), log_n, cols, m31) is not None


def test_wide_fib_trace_definition(oracle):
    # col[i+2] = col[i]^2 + col[i+1]^2: the committed trace root changes with
    # the inputs, and the empty preprocessed tree root is Blake2s("").
    a, b = oracle.wide_fib_inputs(5, 1)
    oracle.prove_wide_fib(oracle.wide_fib_config(5, 10), a, b)
    roots = oracle.last_roots()
    assert roots[0] == hashlib.blake2s(b"").digest()
