"""Generates the golden fixtures of this directory from the CPU oracle.

    python tests/golden/make_golden.py

- wide_fib_8x16.bin: the Wide-Fibonacci proof (log 8 rows, 16 columns,
  blowup 1, default PcsConfig) of the inputs oracle.wide_fib_inputs(8, 2026).
- wide_fib_11x20_m31.bin: the same for log 11 rows, 20 columns, blowup 2,
  line fold step 2, 8 queries, M31-output channel, inputs seed 2027.
- fri_seeded_12.bin: the FRI-heavy proof bytes of oracle.fri_inputs(12, 2028)
  (log 12 column, 70 query draws).
- commit_uneven.json: lifted Merkle root of a small uneven commit (columns
  of log 3..9, blowup 2) of seeded columns.

The oracle is pinned to the reference's own known answers
(reference_kats.json, tests/test_oracle_kats.py); these fixtures freeze its
outputs on larger cases so that both the oracle and the CUDA path are checked
against bytes committed to the repository.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

P = (1 << 31) - 1


def uneven_columns():
    r = np.random.default_rng(2029)
    logs = [int(x) for x in r.integers(3, 10, 24)]
    return logs, [r.integers(0, P, 1 << l, dtype=np.uint32) for l in logs]


def main():
    from oracle import ffi as oracle
    oracle.build()
    a, b = oracle.wide_fib_inputs(8, 2026)
    with open(os.path.join(HERE, "wide_fib_8x16.bin"), "wb") as f:
        f.write(oracle.prove_wide_fib(oracle.wide_fib_config(8, 16), a, b))
    a, b = oracle.wide_fib_inputs(11, 2027)
    cfg = oracle.wide_fib_config(11, 20, log_blowup=2, line_fold_step=2, n_queries=8, m31_channel=True)
    with open(os.path.join(HERE, "wide_fib_11x20_m31.bin"), "wb") as f:
        f.write(oracle.prove_wide_fib(cfg, a, b))
    coords, alphas, queries = oracle.fri_inputs(12, 2028)
    with open(os.path.join(HERE, "fri_seeded_12.bin"), "wb") as f:
        f.write(oracle.fri_prove_seeded(coords, 12, alphas, queries))
    logs, cols = uneven_columns()
    blowup = 2
    init, lg = oracle.canonic_half_coset_root(max(logs) + blowup + 1)
    tw, itw = oracle.precompute_twiddles(init, lg)
    ldes = oracle.evaluate_columns(oracle.interpolate_columns(cols, itw), blowup, tw)
    L = max(logs) + blowup
    root = oracle.merkle_build_layers(ldes, L)[0]
    with open(os.path.join(HERE, "commit_uneven.json"), "w") as f:
        json.dump({"seed": 2029, "log_sizes": logs, "log_blowup": blowup, "lifting_log_size": L,
                   "root": bytes(root.reshape(-1)).hex()}, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
