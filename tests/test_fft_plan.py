"""FFT pass-plan table (host only): validation, round trip and reset.  The
plan is the autotuner's knob; results never depend on it (checked on the GPU
by tests/test_gpu_commit.py)."""
import pytest

from stwo_b200 import ffi, fft_get_plan, fft_set_plan


def test_default_plans():
    assert fft_get_plan(8) == [8]
    assert fft_get_plan(12) == [12]
    assert fft_get_plan(20) == [10, 10]
    assert fft_get_plan(21) == [11, 10]
    assert fft_get_plan(24) == [8, 8, 8]


def test_set_get_reset():
    try:
        fft_set_plan(20, [12, 8])
        assert fft_get_plan(20) == [12, 8]
        fft_set_plan(20, [6, 7, 7])
        assert fft_get_plan(20) == [6, 7, 7]
    finally:
        fft_set_plan(20, [])
    assert fft_get_plan(20) == [10, 10]


@pytest.mark.parametrize("plan", [[2, 18], [13, 7], [10, 9], [0, 20], [3, 3, 3, 3, 8], [1, 19]])
def test_invalid_plans_rejected(plan):
    with pytest.raises(ffi.B200Error):
        fft_set_plan(20, plan)
    assert fft_get_plan(20) == [10, 10]


def test_size_out_of_range():
    with pytest.raises(ffi.B200Error):
        fft_set_plan(31, [11, 10, 10])
    with pytest.raises(ffi.B200Error):
        fft_get_plan(0)
