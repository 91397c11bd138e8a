"""Trace commitment (CommitmentTreeProver path) through the committer object:
per-column, batched and graph-replayed forms, and after autotuning, all give
the oracle's evaluations and Merkle layers byte for byte."""
import os

import numpy as np
import pytest

from stwo_b200 import B200Backend, Committer, DeviceBuffer, DeviceColumn, fft_get_plan, fft_set_plan, layer_to_host

pytestmark = pytest.mark.gpu
P = (1 << 31) - 1


@pytest.fixture(scope="module")
def setup(oracle):
    be = B200Backend()
    r = np.random.default_rng(77)
    logs = [int(x) for x in r.integers(3, 12, 40)] + [3, 11, 12]
    blowup = 2
    init, lg = oracle.canonic_half_coset_root(max(logs) + blowup + 1)
    tw, itw = oracle.precompute_twiddles(init, lg)
    tree = be.precompute_twiddles(init, lg)
    vals = [r.integers(0, P, 1 << l, dtype=np.uint32) for l in logs]
    coeffs = oracle.interpolate_columns(vals, itw)
    ldes = oracle.evaluate_columns(coeffs, blowup, tw)
    L = max(logs) + blowup
    layers = oracle.merkle_build_layers(ldes, L)
    yield dict(be=be, logs=logs, blowup=blowup, tree=tree, vals=vals, coeffs=coeffs, ldes=ldes, layers=layers, L=L)
    for n in set(logs):
        fft_set_plan(n, [])


def buffers(s):
    evals = [DeviceColumn.from_host(v) for v in s["vals"]]
    coeffs = [DeviceColumn(v.size) for v in s["vals"]]
    ldes = [DeviceColumn(v.size << s["blowup"]) for v in s["vals"]]
    return evals, coeffs, ldes


def check(s, coeffs, ldes, layers):
    for k in range(len(s["vals"])):
        assert (coeffs[k].to_host() == s["coeffs"][k]).all(), k
        assert (ldes[k].to_host() == s["ldes"][k]).all(), k
    for k in range(s["L"] + 1):
        assert (layer_to_host(layers[k]) == s["layers"][k]).all(), k


@pytest.mark.parametrize("per_column,graph", [(True, False), (False, False), (False, True)])
def test_commit_forms(setup, per_column, graph):
    s = setup
    cm = Committer(s["logs"], s["blowup"], s["tree"], per_column=per_column, graph=graph)
    assert cm.lifting_log_size == s["L"]
    evals, coeffs, ldes = buffers(s)
    layers = cm.new_layers()
    for _ in range(2):  # the second call replays the graph
        cm.commit(evals, coeffs, ldes, layers)
        check(s, coeffs, ldes, layers)
    if graph:  # new buffers: recaptured
        evals2, coeffs2, ldes2 = buffers(s)
        layers2 = cm.new_layers()
        cm.commit(evals2, coeffs2, ldes2, layers2)
        check(s, coeffs2, ldes2, layers2)
    cm.close()


@pytest.mark.parametrize("per_column", [False, True])
def test_commit_from_host(setup, per_column):
    # the columns start in (pinned) host memory and are copied size group by
    # size group while earlier groups are transformed; same bytes as commit()
    import torch

    s = setup
    cm = Committer(s["logs"], s["blowup"], s["tree"], per_column=per_column)
    pinned = []
    for v in s["vals"]:
        t = torch.empty(v.size, dtype=torch.int32).pin_memory()
        t.numpy().view(np.uint32)[:] = v
        pinned.append(t)
    evals = [DeviceColumn(v.size) for v in s["vals"]]
    coeffs = [DeviceColumn(v.size) for v in s["vals"]]
    ldes = [DeviceColumn(v.size << s["blowup"]) for v in s["vals"]]
    layers = cm.new_layers()
    for _ in range(2):  # the second call reuses the copy stream and events
        cm.commit_from_host([t.data_ptr() for t in pinned], evals, coeffs, ldes, layers)
        for e, v in zip(evals, s["vals"]):
            assert (e.to_host() == v).all()
        check(s, coeffs, ldes, layers)
    cm.close()


def test_autotune_and_cache(setup, tmp_path):
    s = setup
    cm = Committer(s["logs"], s["blowup"], s["tree"], graph=True)
    evals, coeffs, ldes = buffers(s)
    layers = cm.new_layers()
    cache = str(tmp_path / "plans.txt")
    cm.autotune(evals, coeffs, ldes, cache_path=cache, reps=2)
    lines = open(cache).read().split("\n")
    groups = {}
    for l in s["logs"]:
        groups[l] = groups.get(l, 0) + 1
    entries = {}
    for line in filter(None, lines):
        n, k, plan = line.split()
        entries[(int(n), int(k))] = [int(x) for x in plan.split(",")]
    assert set(entries) == set(groups.items())
    for (n, _), plan in entries.items():
        assert sum(plan) == n and fft_get_plan(n) == plan
    cm.commit(evals, coeffs, ldes, layers)
    check(s, coeffs, ldes, layers)
    # a planted cache entry is applied without timing
    n0 = max(s["logs"])
    entries[(n0, groups[n0])] = [3, n0 - 3]
    with open(cache, "w") as f:
        for (n, k), plan in entries.items():
            f.write(f"{n} {k} {','.join(map(str, plan))}\n")
    cm.autotune(evals, coeffs, ldes, cache_path=cache, reps=2)
    assert fft_get_plan(n0) == [3, n0 - 3]
    cm.commit(evals, coeffs, ldes, layers)
    check(s, coeffs, ldes, layers)
    cm.close()


def test_committer_rejects_bad_shapes(setup):
    from stwo_b200 import ffi
    s = setup
    with pytest.raises(ffi.B200Error):
        Committer([], 1, s["tree"])
    with pytest.raises(ffi.B200Error):
        Committer([30], 1, s["tree"])
