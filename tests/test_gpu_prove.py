"""End-to-end parity: Wide-Fibonacci proofs from the B200 prover are
byte-identical to the oracle's (stwo SimdBackend restatement) and the
restated stwo verifier accepts them."""
import numpy as np
import pytest

from stwo_b200 import DeviceColumn, WideFibProver, wide_fib_config

pytestmark = pytest.mark.gpu


CASES = [
    # (log_n, n_cols, log_blowup, line_fold_step, log_last_layer, n_queries, m31)
    (4, 100, 1, 1, 0, 3, False),
    (5, 8, 1, 1, 0, 3, True),
    (6, 3, 1, 1, 0, 3, False),
    (8, 100, 1, 1, 0, 3, False),
    (10, 16, 2, 1, 0, 5, False),
    (11, 20, 1, 2, 0, 8, False),
    (12, 32, 1, 3, 1, 16, True),
    (14, 100, 1, 1, 0, 3, False),
    (16, 64, 1, 1, 0, 3, False),
    # the interpolation's last pass fused with the evaluation's first
    # (layers 10..19 at log 20, 11..20 at log 21; blowup 1), and the two
    # separate passes at blowup 2
    (20, 8, 1, 1, 0, 3, False),
    (20, 4, 2, 1, 0, 3, False),
    (21, 4, 1, 1, 0, 3, False),
]


@pytest.mark.parametrize("log_n,cols,blowup,step,last,nq,m31", CASES)
def test_wide_fib_proof_bytes_match_oracle(oracle, log_n, cols, blowup, step, last, nq, m31):
    a, b = oracle.wide_fib_inputs(log_n, 1000 + log_n)
    ocfg = oracle.wide_fib_config(log_n, cols, log_blowup=blowup, line_fold_step=step,
                                  log_last_layer_degree_bound=last, n_queries=nq, m31_channel=m31)
    ref = oracle.prove_wide_fib(ocfg, a, b)
    prover = WideFibProver(wide_fib_config(log_n, cols, log_blowup=blowup, line_fold_step=step,
                                           log_last_layer_degree_bound=last, n_queries=nq, m31_channel=m31))
    got = prover.prove(DeviceColumn.from_host(a), DeviceColumn.from_host(b))
    assert len(got) == len(ref)
    if got != ref:
        first = next(i for i in range(len(ref)) if got[i] != ref[i])
        pytest.fail(f"proof bytes differ first at offset {first} of {len(ref)}")
    assert oracle.verify_wide_fib(got, log_n, cols, m31) is None


@pytest.mark.parametrize("pow_bits,last", [(0, 0), (20, 0), (10, 5), (10, 6)])
def test_proof_of_work_and_last_layer_forms(oracle, pow_bits, last):
    # The last-layer interpolation, the proof-of-work prefix and the first
    # grind batch (2^16 nonces) run on the device for last layers of up to 64
    # values.  At 20 bits that batch misses with probability ~0.94 and the
    # host continues the search; a last layer of 2^7 values stays on the host.
    log_n, cols = 10, 8
    a, b = oracle.wide_fib_inputs(log_n, 500 + pow_bits + last)
    ocfg = oracle.wide_fib_config(log_n, cols, pow_bits=pow_bits, log_last_layer_degree_bound=last)
    ref = oracle.prove_wide_fib(ocfg, a, b)
    prover = WideFibProver(wide_fib_config(log_n, cols, pow_bits=pow_bits, log_last_layer_degree_bound=last))
    got = prover.prove(DeviceColumn.from_host(a), DeviceColumn.from_host(b))
    assert got == ref
    assert prover.prove(DeviceColumn.from_host(a), DeviceColumn.from_host(b)) == ref


@pytest.mark.parametrize("plan", [[6, 10], [8, 8], [7, 9], [4, 6, 6]])
def test_proof_under_other_pass_splits(oracle, plan):
    # The prover's transforms follow the process-wide plan table: the log-16
    # trace transforms under splits other than the default [10, 6] --
    # contiguous 6..8-layer warp passes, strided passes at layer offsets 6..8,
    # three passes -- give the oracle's proof bytes.
    from stwo_b200 import fft_get_plan, fft_set_plan
    log_n, cols = 16, 8
    a, b = oracle.wide_fib_inputs(log_n, 900 + sum(plan))
    ref = oracle.prove_wide_fib(oracle.wide_fib_config(log_n, cols), a, b)
    old = fft_get_plan(log_n)
    fft_set_plan(log_n, plan)
    try:
        prover = WideFibProver(wide_fib_config(log_n, cols))
        assert prover.prove(DeviceColumn.from_host(a), DeviceColumn.from_host(b)) == ref
    finally:
        fft_set_plan(log_n, old)


def test_prover_reuse_is_deterministic(oracle):
    # Resident buffers are reused across proofs: a second proof of other
    # inputs, then the first inputs again, reproduce the oracle bytes.
    log_n, cols = 9, 24
    prover = WideFibProver(wide_fib_config(log_n, cols))
    ins = [oracle.wide_fib_inputs(log_n, s) for s in (1, 2)]
    outs = [prover.prove(DeviceColumn.from_host(a), DeviceColumn.from_host(b)) for a, b in ins + ins[:1]]
    assert outs[0] == outs[2] != outs[1]
    assert outs[1] == oracle.prove_wide_fib(oracle.wide_fib_config(log_n, cols), *ins[1])


def test_invalid_config_rejected():
    from stwo_b200 import ffi
    with pytest.raises(ffi.B200Error):
        WideFibProver(wide_fib_config(2, 100))
    with pytest.raises(ffi.B200Error):
        WideFibProver(wide_fib_config(8, 2))


def test_phase_timing_does_not_change_proofs(oracle):
    # The timed path records CUDA events between phases; proofs must be
    # unchanged and every phase must have been timed.
    import ctypes as C
    from stwo_b200 import ffi
    log_n, cols = 12, 100
    a, b = oracle.wide_fib_inputs(log_n, 77)
    ref = oracle.prove_wide_fib(oracle.wide_fib_config(log_n, cols), a, b)
    prover = WideFibProver(wide_fib_config(log_n, cols))
    da, db = DeviceColumn.from_host(a), DeviceColumn.from_host(b)
    ffi.call("stwo_b200_prover_set_timing", prover.handle, C.c_int(1))
    for _ in range(4):
        assert prover.prove(da, db) == ref
    ms = (C.c_double * 14)()
    n = C.c_uint32()
    ffi.call("stwo_b200_prover_phase_times", prover.handle, ms, C.c_uint32(14), C.byref(n))
    assert n.value == 4
    assert all(x > 0 for x in ms)


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("log_n", [12, 16, 20])
def test_prove_from_host_columns(oracle, pinned, log_n):
    # host inputs (pageable numpy, or page-locked memory from the library):
    # copied chunk by chunk by the prover, the same proof bytes.  From log 16
    # the interpolation is split in passes and its first pass runs chunk by
    # chunk as the trace rows are generated; at log 20 its last pass runs
    # fused with the evaluation.
    import ctypes as C
    from stwo_b200 import ffi
    cols = 24 if log_n < 20 else 6
    a, b = oracle.wide_fib_inputs(log_n, 55)
    ref = oracle.prove_wide_fib(oracle.wide_fib_config(log_n, cols), a, b)
    prover = WideFibProver(wide_fib_config(log_n, cols))
    if not pinned:
        assert prover.prove_host(a, b) == ref
        assert prover.prove(DeviceColumn.from_host(a), DeviceColumn.from_host(b)) == ref  # device path after
        assert prover.prove_host(a, b) == ref
        return
    hp = C.c_void_p()
    ffi.call("stwo_b200_host_alloc", C.c_size_t(8 << log_n), C.byref(hp))
    try:
        host = np.ctypeslib.as_array((C.c_uint32 * (2 << log_n)).from_address(hp.value))
        host[: 1 << log_n] = a
        host[1 << log_n:] = b
        buf = (C.c_uint8 * (1 << 22))()
        for _ in range(2):
            n = prover.prove_host_into(hp.value, hp.value + (4 << log_n), buf, len(buf))
            assert C.string_at(buf, n) == ref
    finally:
        ffi.call("stwo_b200_host_free", hp)
