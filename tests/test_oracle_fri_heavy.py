"""Oracle FRI-heavy restatement (one secure column, seeded alphas, folds to a
single value, 70 queries): its bytes parse as a FriProof whose roots and last
value agree with the oracle's fold and Merkle primitives applied step by step
(each of which is pinned by the KATs and naive-evaluation tests)."""
import struct

import numpy as np
import pytest


def parse(b, log_n):
    off = 0

    def u64():
        nonlocal off
        v = struct.unpack_from("<Q", b, off)[0]
        off += 8
        return v

    def take(n):
        nonlocal off
        v = b[off:off + n]
        off += n
        return v

    def layer():
        nw = u64()
        wit = [np.frombuffer(take(16), np.uint32) for _ in range(nw)]
        nn = u64()
        nodes = [take(32) for _ in range(nn)]
        return dict(witness=wit, nodes=nodes, root=take(32))

    first = layer()
    n_inner = u64()
    inner = [layer() for _ in range(n_inner)]
    assert u64() == 1
    last = np.frombuffer(take(16), np.uint32)
    assert off == len(b)
    return first, inner, last


@pytest.mark.parametrize("log_n,m31", [(2, False), (3, True), (6, False), (11, False), (12, True)])
def test_fri_heavy_structure(oracle, log_n, m31):
    coords, alphas, queries = oracle.fri_inputs(log_n, 100 + log_n, 70)
    b = oracle.fri_prove_seeded(coords, log_n, alphas, queries, m31)
    first, inner, last = parse(b, log_n)
    assert len(inner) == log_n - 1
    init, lg = oracle.canonic_half_coset_root(log_n + 1)
    tw, itw = oracle.precompute_twiddles(init, lg)
    assert first["root"] == bytes(oracle.merkle_build_layers(coords, log_n, m31)[0][0])
    cur = oracle.fold_circle_into_line([np.zeros(1 << (log_n - 1), np.uint32)] * 4, coords, itw, alphas[0])
    for k in range(1, log_n):
        assert inner[k - 1]["root"] == bytes(oracle.merkle_build_layers(cur, log_n - k, m31)[0][0]), k
        cur = oracle.fold_line(cur, itw, alphas[k], 1)
    assert [int(c[0]) for c in cur] == [int(x) for x in last]
    # witnesses: one sibling per query whose pair partner is not queried
    q = sorted(set(int(x) for x in queries))
    pairs = {}
    for p in q:
        pairs.setdefault(p >> 1, set()).add(p)
    assert len(first["witness"]) == sum(1 for s in pairs.values() if len(s) == 1)


def test_fri_heavy_rejects_bad_queries(oracle):
    coords, alphas, _ = oracle.fri_inputs(5, 1, 4)
    with pytest.raises(Exception):
        oracle.fri_prove_seeded(coords, 5, alphas, np.array([1 << 5], np.uint64))
