"""stwo_b200 -- B200-native (sm_100a) backend for stwo's commit + FRI path.

The compute lives in ``libstwo_b200.so`` (hand-written CUDA kernels behind the
flat C ABI of ``include/stwo_b200.h``); this package is its Python view.
"""
from . import ffi
from .prover import (ProveServer, SeededFriProver, WideFibConfig, WideFibProver, prover_footprint,
                     wide_fib_config)
from .backend import (B200Backend, Committer, DeviceBuffer, DeviceColumn, SecureColumn, TwiddleTree,
                      canonic_half_coset, fft_get_plan, fft_set_plan, layer_to_host, sync)

__all__ = ["ffi", "ProveServer", "prover_footprint", "SeededFriProver", "WideFibConfig", "WideFibProver", "wide_fib_config", "B200Backend", "Committer", "fft_get_plan", "fft_set_plan", "DeviceBuffer", "DeviceColumn", "SecureColumn", "TwiddleTree",
           "canonic_half_coset", "layer_to_host", "sync"]
