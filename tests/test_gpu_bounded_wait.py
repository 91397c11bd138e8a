"""The bounded device waits of the column-streaming kernels give up cleanly.

The composition and quotient kernels stream columns through a shared-memory
ring whose stages complete on mbarriers; every wait on them is bounded.  Here
the consumers' bound is set to zero polls, so the first stage wait of every
block runs out: the block sets the prover's error flag, the producer waits for
its copies already in flight and leaves, and the prove returns
STWO_B200_ETIMEOUT with a message.  Nothing faults, and the same prover then
proves the same inputs with the default bound, byte for byte as the oracle.
"""
import pytest

from stwo_b200 import DeviceColumn, WideFibProver, ffi, wide_fib_config

pytestmark = pytest.mark.gpu
ETIMEOUT = -4


@pytest.mark.parametrize("log_n,cols", [(12, 100), (16, 24)])
def test_stream_wait_timeout_reports_and_recovers(oracle, log_n, cols):
    a, b = oracle.wide_fib_inputs(log_n, 4242 + log_n)
    ref = oracle.prove_wide_fib(oracle.wide_fib_config(log_n, cols), a, b)
    prover = WideFibProver(wide_fib_config(log_n, cols))
    da, db = DeviceColumn.from_host(a), DeviceColumn.from_host(b)
    assert prover.prove(da, db) == ref
    prover.set_stream_spin(0)
    with pytest.raises(ffi.B200Error) as e:
        prover.prove(da, db)
    assert e.value.code == ETIMEOUT
    assert "column stream" in str(e.value)
    prover.set_stream_spin(WideFibProver.STREAM_SPIN_DEFAULT)
    assert prover.prove(da, db) == ref
    assert prover.prove(da, db) == ref
    prover.close()
