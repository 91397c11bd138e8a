"""Prover footprint (host-only): the allocation arithmetic of a prover's init,
used by the server's HBM admission."""
from stwo_b200 import prover_footprint, wide_fib_config


def test_footprint_grows_with_shape():
    f = {(ln, nc): prover_footprint(wide_fib_config(ln, nc)) for ln in (8, 14, 20) for nc in (16, 100, 256)}
    for ln in (8, 14, 20):
        assert f[(ln, 16)] < f[(ln, 100)] < f[(ln, 256)]
    for nc in (16, 100, 256):
        assert f[(8, nc)] < f[(14, nc)] < f[(20, nc)]


def test_footprint_covers_trace_buffers():
    ln, nc = 20, 100
    fp = prover_footprint(wide_fib_config(ln, nc))
    # coefficients (2^20) + evaluations (2^21) of every column, 4 bytes a word
    assert fp > 4 * nc * ((1 << ln) + (1 << (ln + 1)))
    assert fp < 4 << 30
