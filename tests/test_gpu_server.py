"""Serving: requests of mixed shapes submitted concurrently to the prove
server (3 slots, an HBM budget small enough to force evictions) each give the
proof the same request gives alone on its own prover (and the oracle's, for
the small ones); the server overlapped requests and reused and evicted
resident provers."""
import threading

import numpy as np
import pytest

from stwo_b200 import DeviceColumn, ProveServer, WideFibProver, ffi, prover_footprint, wide_fib_config

pytestmark = pytest.mark.gpu

SHAPES = [(6, 8), (7, 20), (6, 70), (8, 12), (6, 8), (7, 100), (5, 3), (9, 40), (7, 20), (6, 130), (8, 12),
          (6, 8), (10, 16), (7, 64), (5, 3), (9, 40)]


def inputs(oracle, log_n, seed):
    return oracle.wide_fib_inputs(log_n, seed)


def test_server_mix_equals_alone(oracle):
    reqs = [(ln, nc, *inputs(oracle, ln, 500 + i)) for i, (ln, nc) in enumerate(SHAPES)]
    alone = []
    for ln, nc, a, b in reqs:
        p = WideFibProver(wide_fib_config(ln, nc))
        alone.append(p.prove(DeviceColumn.from_host(a), DeviceColumn.from_host(b)))
        p.close()
    for (ln, nc, a, b), pr in zip(reqs, alone):
        if ln <= 7 and nc <= 20:
            assert pr == oracle.prove_wide_fib(oracle.wide_fib_config(ln, nc), a, b)
    # budget: room for about three of the larger residents
    big = max(prover_footprint(wide_fib_config(ln, ((nc + 63) // 64) * 64)) + (8 << ln) for ln, nc in SHAPES)
    srv = ProveServer(3 * big + (64 << 20), slots=3)
    tickets = [None] * len(reqs)

    def submit(idx):
        for i in idx:
            ln, nc, a, b = reqs[i]
            tickets[i] = srv.submit(wide_fib_config(ln, nc), a, b)

    ths = [threading.Thread(target=submit, args=(range(k, len(reqs), 3),)) for k in range(3)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    results = [srv.wait(t) for t in tickets]
    for i, ((proof, times), ref) in enumerate(zip(results, alone)):
        assert proof == ref, SHAPES[i]
        assert times["latency_ms"] >= times["service_ms"] > 0
    st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["max_running"] >= 2
    assert st["provers_reused"] >= 1
    assert st["provers_evicted"] >= 1
    srv.close()


def test_server_rejects_oversized_and_unknown(oracle):
    srv = ProveServer(64 << 20, slots=1)
    a, b = inputs(oracle, 16, 1)
    with pytest.raises(ffi.B200Error):
        srv.submit(wide_fib_config(16, 256), a, b)
    with pytest.raises(ffi.B200Error):
        srv.wait(12345)
    srv.close()


def test_prove_cols_matches_exact_width(oracle):
    ln = 7
    wide = WideFibProver(wide_fib_config(ln, 64))
    for nc in (3, 17, 64):
        a, b = inputs(oracle, ln, 900 + nc)
        exact = WideFibProver(wide_fib_config(ln, nc))
        da, db = DeviceColumn.from_host(a), DeviceColumn.from_host(b)
        assert wide.prove_cols(da, db, nc) == exact.prove(da, db)
        exact.close()
    with pytest.raises(ffi.B200Error):
        wide.prove_cols(da, db, 65)
    wide.close()
