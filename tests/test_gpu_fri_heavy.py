"""FRI-heavy path on the GPU (one secure column, seeded alphas, every layer
folded by 2 to a single value, Blake2s tree per layer, decommitments of the
query positions): byte-identical to the oracle's FriProof bytes."""
import numpy as np
import pytest

from stwo_b200 import B200Backend, DeviceColumn, SeededFriProver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def be():
    return B200Backend()


def tree_for(be, oracle, log_n):
    init, lg = oracle.canonic_half_coset_root(log_n + 1)
    return be.precompute_twiddles(init, lg)


@pytest.mark.parametrize("log_n,m31", [(2, False), (3, False), (4, True), (5, False), (8, False), (12, True),
                                       (16, False), (19, False)])
def test_fri_heavy_matches_oracle(be, oracle, log_n, m31):
    coords, alphas, queries = oracle.fri_inputs(log_n, 300 + log_n, 70)
    ref = oracle.fri_prove_seeded(coords, log_n, alphas, queries, m31)
    fp = SeededFriProver(log_n, tree_for(be, oracle, log_n), m31=m31)
    dev = [DeviceColumn.from_host(c) for c in coords]
    assert fp.prove(dev, alphas, queries) == ref
    fp.close()


def test_fri_heavy_edge_queries_and_reuse(be, oracle):
    log_n = 10
    fp = SeededFriProver(log_n, tree_for(be, oracle, log_n))
    for seed, queries in [(1, [0]), (2, [(1 << log_n) - 1]), (3, [4, 5]), (4, [0, 1, 2, 3, 1022, 1023]),
                          (5, list(range(0, 1 << log_n, 7)))]:
        coords, alphas, _ = oracle.fri_inputs(log_n, seed, 1)
        q = np.array(queries, np.uint64)
        ref = oracle.fri_prove_seeded(coords, log_n, alphas, q)
        dev = [DeviceColumn.from_host(c) for c in coords]
        assert fp.prove(dev, alphas, q) == ref, queries
    fp.close()


def test_fri_heavy_rejects_unsorted_queries(be, oracle):
    from stwo_b200 import ffi
    log_n = 6
    fp = SeededFriProver(log_n, tree_for(be, oracle, log_n))
    coords, alphas, _ = oracle.fri_inputs(log_n, 9, 1)
    dev = [DeviceColumn.from_host(c) for c in coords]
    with pytest.raises(ffi.B200Error):
        fp.prove(dev, alphas, np.array([5, 3], np.uint64))
    with pytest.raises(ffi.B200Error):
        fp.prove(dev, alphas, np.array([1 << log_n], np.uint64))
    fp.close()
