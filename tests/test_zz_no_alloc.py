"""FriOps::decompose through the no-allocation entry point.

stwo_b200_decompose_noalloc serves callers that cannot let the library
allocate device memory while they run (their device memory is divided up
front, e.g. by a prover service's admission controller, or owned by their own
runtime).  Its reduction scratch is a fixed device array instead of a pool
allocation.  This checks, through the C ABI, that it returns exactly what the
allocating entry point stwo_b200_decompose returns, on calls in a row of
different sizes: each call reuses the shared scratch the previous one left
behind.
Collected last so a stop-at-first-failure run has already run the rest.
"""
import ctypes as C

import numpy as np
import pytest

from stwo_b200 import B200Backend, SecureColumn, ffi
from stwo_b200.backend import _ptr_array

pytestmark = pytest.mark.gpu
P = (1 << 31) - 1


def _decompose_noalloc(ev: SecureColumn):
    out = SecureColumn.empty(ev.length)
    lam = (C.c_uint32 * 4)()
    ffi.call("stwo_b200_decompose_noalloc", _ptr_array(ev.cols), C.c_uint32(ev.cols[0].log_size),
             _ptr_array(out.cols), lam, None)
    return out, np.array(list(lam), np.uint32)


def test_decompose_noalloc_matches_allocating_entry_point():
    be = B200Backend()
    rng = np.random.default_rng(2024)
    # large then small (the small call reads only partials it wrote itself),
    # sizes below 16 elements (no reduction blocks with data, lambda 0), then
    # small then large again (the large call overwrites every partial it reads)
    for log_n in (20, 12, 0, 3, 4, 5, 21):
        coords = [rng.integers(0, P, 1 << log_n, dtype=np.uint32) for _ in range(4)]
        ev = SecureColumn.from_host(coords)
        g_ref, lam_ref = be.decompose(ev)
        g, lam = _decompose_noalloc(ev)
        assert (lam == lam_ref).all(), log_n
        for got, ref in zip(g.to_host(), g_ref.to_host()):
            assert (got == ref).all(), log_n


def test_decompose_noalloc_rejects_sizes_beyond_maximum():
    ev = SecureColumn.from_host([np.zeros(16, np.uint32) for _ in range(4)])
    lam = (C.c_uint32 * 4)()
    with pytest.raises(ffi.B200Error, match="exceeds the maximum"):
        ffi.call("stwo_b200_decompose_noalloc", _ptr_array(ev.cols), C.c_uint32(31), _ptr_array(ev.cols), lam, None)
