"""Digests of the oracle's outputs at the benchmarked sizes.

    python tests/golden/make_full_size_digests.py

Writes full_size_digests.json: for each benchmark configuration, on the same
seeded inputs bench.py generates, the oracle's Merkle root (commits) or the
SHA-256 of its proof bytes (proofs):

- commit_plain: 32 columns of log 16 (numpy PCG64 seed 1001), natural order,
  blowup 1, lifted Blake2s tree of log 17;
- wide_fib_prove: 100 columns x 2^20 rows (seed 2), default PcsConfig;
- commit_uneven: 512 columns, log sizes U{12..22} (seed 3), values seed 1003,
  blowup 2, lifted tree of log 24;
- fri_heavy: one QM31 column of log 24 (seed 4), 70 query draws.

bench.py compares its roots and proofs at these sizes with these digests, so
that a bench line states bit-exactness without running the oracle for
minutes.  tests/test_golden.py checks the cheap entries against the oracle
again; tests/test_gpu_full_size.py checks every one of them on the GPU
against a fresh oracle run.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

P = (1 << 31) - 1


def commit_plain_columns():
    r = np.random.default_rng(1 + 1000)
    return [16] * 32, [r.integers(0, P, 1 << 16, dtype=np.uint32) for _ in range(32)]


def commit_uneven_columns():
    logs = [int(x) for x in np.random.default_rng(3).integers(12, 23, 512)]
    r = np.random.default_rng(3 + 1000)
    return logs, [r.integers(0, P, 1 << l, dtype=np.uint32) for l in logs]


def wide_fib_columns():
    r = np.random.default_rng(2)
    return r.integers(0, P, 1 << 20, dtype=np.uint32), r.integers(0, P, 1 << 20, dtype=np.uint32)


def commit_root(oracle, logs, cols, blowup, natural):
    L = max(logs) + blowup
    init, lg = oracle.canonic_half_coset_root(L + 1)
    tw, itw = oracle.precompute_twiddles(init, lg)
    src = [oracle.bit_reverse(c) for c in cols] if natural else cols
    coeffs = oracle.interpolate_columns(src, itw)
    evals = oracle.evaluate_columns(coeffs, blowup, tw)
    del coeffs
    leaves = oracle.merkle_build_leaves(evals, L)
    del evals
    layer = leaves
    while layer.shape[0] > 1:
        layer = oracle.merkle_next_layer(layer)
    return bytes(layer[0]).hex()


def main():
    from oracle import ffi as oracle
    oracle.build()
    out = {}
    logs, cols = commit_plain_columns()
    out["commit_plain_root"] = commit_root(oracle, logs, cols, 1, True)
    a, b = wide_fib_columns()
    proof = oracle.prove_wide_fib(oracle.wide_fib_config(20, 100), a, b)
    out["wide_fib_prove_sha256"] = hashlib.sha256(proof).hexdigest()
    out["wide_fib_prove_bytes"] = len(proof)
    coords, alphas, queries = oracle.fri_inputs(24, 4, 70)
    fri = oracle.fri_prove_seeded(coords, 24, alphas, queries)
    out["fri_heavy_sha256"] = hashlib.sha256(fri).hexdigest()
    out["fri_heavy_bytes"] = len(fri)
    logs, cols = commit_uneven_columns()
    order = sorted(range(len(logs)), key=lambda i: logs[i])
    out["commit_uneven_root"] = commit_root(oracle, [logs[i] for i in order], [cols[i] for i in order], 2, False)
    with open(os.path.join(HERE, "full_size_digests.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
