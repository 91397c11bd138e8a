"""Committed golden vectors.

reference_kats.json holds known answers transcribed from the reference's own
unit tests; the oracle must reproduce every one.  The .bin/.json fixtures are
oracle outputs on fixed seeds (tests/golden/make_golden.py): the oracle must
still reproduce them byte for byte, the oracle verifier must accept the
proofs, and on the GPU the B200 path must produce the same bytes.
"""
import hashlib
import json
import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
P = (1 << 31) - 1

# (fixture, log_n, n_cols, log_blowup, line_fold_step, n_queries, m31, seed)
WIDE_FIB = [("wide_fib_8x16.bin", 8, 16, 1, 1, 3, False, 2026),
            ("wide_fib_11x20_m31.bin", 11, 20, 2, 2, 8, True, 2027)]
FRI = ("fri_seeded_12.bin", 12, 2028)


def _read(name, mode="rb"):
    with open(os.path.join(HERE, name), mode) as f:
        return f.read()


def _felt(v):
    return P - int(v[2:]) if isinstance(v, str) else int(v)


def _uneven(spec):
    r = np.random.default_rng(spec["seed"])
    logs = [int(x) for x in r.integers(3, 10, len(spec["log_sizes"]))]
    assert logs == spec["log_sizes"]
    return logs, [r.integers(0, P, 1 << l, dtype=np.uint32) for l in logs]


def test_reference_kats(oracle):
    k = json.loads(_read("reference_kats.json", "r"))
    for e in k["blake2s"]:
        data = bytes.fromhex(e["input_hex"])
        assert oracle.blake2s(data).hex() == e["digest"] == hashlib.blake2s(data).hexdigest()
    for e in k["channel_mix_u64"]:
        c = oracle.Channel()
        c.mix_u64(int(e["value"], 16))
        assert c.digest.hex() == e["digest"]
        c2 = oracle.Channel()
        c2.mix_u32s(e["equals_mix_u32s"])
        assert c2.digest.hex() == e["digest"]
    for e in k["channel_mix_u32s"]:
        c = oracle.Channel()
        c.mix_u32s(e["words"])
        assert c.digest.hex() == e["digest"]
    for e in k["channel_draw_counts"]:
        c = oracle.Channel()
        c.draw_u32s()
        assert c.n_draws == e["after_draw_u32s"]
        c.draw_secure_felts(9)
        assert c.n_draws == e["after_draw_secure_felts_9"]
    for e in k["qm31_mul"]:
        prod = tuple(_felt(v) for v in e["product"])
        assert oracle.qm31_mul(e["a"], e["b"]) == prod
        assert oracle.qm31_mul(prod, oracle.qm31_inv(e["b"])) == tuple(e["a"])
    for e in k["cm31_mul"]:
        prod = tuple(_felt(v) for v in e["product"]) + (0, 0)
        assert oracle.qm31_mul(e["a"] + [0, 0], e["b"] + [0, 0]) == prod


@pytest.mark.parametrize("name,log_n,cols,blowup,step,nq,m31,seed", WIDE_FIB)
def test_oracle_reproduces_wide_fib_fixture(oracle, name, log_n, cols, blowup, step, nq, m31, seed):
    ref = _read(name)
    a, b = oracle.wide_fib_inputs(log_n, seed)
    cfg = oracle.wide_fib_config(log_n, cols, log_blowup=blowup, line_fold_step=step, n_queries=nq,
                                 m31_channel=m31)
    assert oracle.prove_wide_fib(cfg, a, b) == ref
    assert oracle.verify_wide_fib(ref, log_n, cols, m31) is None


def test_oracle_reproduces_fri_fixture(oracle):
    name, log_n, seed = FRI
    coords, alphas, queries = oracle.fri_inputs(log_n, seed)
    assert oracle.fri_prove_seeded(coords, log_n, alphas, queries) == _read(name)


def test_oracle_reproduces_uneven_commit_fixture(oracle):
    spec = json.loads(_read("commit_uneven.json", "r"))
    logs, cols = _uneven(spec)
    init, lg = oracle.canonic_half_coset_root(max(logs) + spec["log_blowup"] + 1)
    tw, itw = oracle.precompute_twiddles(init, lg)
    ldes = oracle.evaluate_columns(oracle.interpolate_columns(cols, itw), spec["log_blowup"], tw)
    root = oracle.merkle_build_layers(ldes, spec["lifting_log_size"])[0]
    assert bytes(root.reshape(-1)).hex() == spec["root"]


def test_oracle_reproduces_full_size_digests(oracle):
    # full_size_digests.json (make_full_size_digests.py) is what bench.py
    # compares its full-size results with; the quick entries are re-derived
    # here, the 512-column commit root on the GPU suite's full-size test.
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", os.path.join(HERE, "make_full_size_digests.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    d = json.loads(_read("full_size_digests.json", "r"))
    logs, cols = mk.commit_plain_columns()
    assert mk.commit_root(oracle, logs, cols, 1, True) == d["commit_plain_root"]
    a, b = mk.wide_fib_columns()
    proof = oracle.prove_wide_fib(oracle.wide_fib_config(20, 100), a, b)
    assert (hashlib.sha256(proof).hexdigest(), len(proof)) == (d["wide_fib_prove_sha256"], d["wide_fib_prove_bytes"])
    coords, alphas, queries = oracle.fri_inputs(24, 4, 70)
    fri = oracle.fri_prove_seeded(coords, 24, alphas, queries)
    assert (hashlib.sha256(fri).hexdigest(), len(fri)) == (d["fri_heavy_sha256"], d["fri_heavy_bytes"])


@pytest.mark.gpu
@pytest.mark.parametrize("name,log_n,cols,blowup,step,nq,m31,seed", WIDE_FIB)
def test_gpu_wide_fib_matches_fixture(oracle, name, log_n, cols, blowup, step, nq, m31, seed):
    from stwo_b200 import DeviceColumn, WideFibProver, wide_fib_config
    a, b = oracle.wide_fib_inputs(log_n, seed)
    prover = WideFibProver(wide_fib_config(log_n, cols, log_blowup=blowup, line_fold_step=step, n_queries=nq,
                                           m31_channel=m31))
    assert prover.prove(DeviceColumn.from_host(a), DeviceColumn.from_host(b)) == _read(name)


@pytest.mark.gpu
def test_gpu_fri_matches_fixture(oracle):
    from stwo_b200 import B200Backend, DeviceColumn, SeededFriProver
    name, log_n, seed = FRI
    coords, alphas, queries = oracle.fri_inputs(log_n, seed)
    tree = B200Backend().precompute_twiddles(*oracle.canonic_half_coset_root(log_n + 1))
    fp = SeededFriProver(log_n, tree)
    assert fp.prove([DeviceColumn.from_host(c) for c in coords], alphas, queries) == _read(name)
    fp.close()


@pytest.mark.gpu
def test_gpu_uneven_commit_matches_fixture(oracle):
    from stwo_b200 import B200Backend, Committer, DeviceColumn, layer_to_host
    spec = json.loads(_read("commit_uneven.json", "r"))
    logs, cols = _uneven(spec)
    be = B200Backend()
    tree = be.precompute_twiddles(*oracle.canonic_half_coset_root(max(logs) + spec["log_blowup"] + 1))
    cm = Committer(logs, spec["log_blowup"], tree)
    assert cm.lifting_log_size == spec["lifting_log_size"]
    evals = [DeviceColumn.from_host(c) for c in cols]
    coeffs = [DeviceColumn(c.size) for c in cols]
    ldes = [DeviceColumn(c.size << spec["log_blowup"]) for c in cols]
    layers = cm.new_layers()
    cm.commit(evals, coeffs, ldes, layers)
    assert bytes(layer_to_host(layers[0]).reshape(-1)).hex() == spec["root"]
    cm.close()
