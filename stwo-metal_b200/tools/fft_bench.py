"""FFT benchmark of the trace transforms: interpolate n_cols x 2^log_n
bit-reversed evaluations, then evaluate the coefficients on the blowup-1
domain, through the batched C ABI (the calls the prover makes).  Prints the
time of each per iteration: host clock between device synchronisations,
averaged over the iterations after the second.  Element-layers count every
element of every butterfly layer: log_n layers for both, since evaluate
transforms each of the two half-size subdomains with the layers below log_n.

    python stwo-metal_b200/tools/fft_bench.py [log_n=20] [n_cols=64] [iters=10]
"""
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402

from stwo_b200 import B200Backend, DeviceColumn  # noqa: E402
from stwo_b200.backend import sync  # noqa: E402

P = (1 << 31) - 1


def main():
    log_n = int(sys.argv[1]) if len(sys.argv) > 1 else 20
    n_cols = int(sys.argv[2]) if len(sys.argv) > 2 else 64
    iters = int(sys.argv[3]) if len(sys.argv) > 3 else 10
    be = B200Backend()
    lg = log_n + 1
    tree = be.precompute_twiddles(1 << (31 - (lg + 2)), lg)  # CanonicCoset(lg + 1).half_coset
    host = np.random.default_rng(1).integers(0, P, 1 << log_n, dtype=np.uint32)
    evals = [DeviceColumn.from_host(host) for _ in range(n_cols)]
    coeffs = [DeviceColumn(1 << log_n) for _ in range(n_cols)]
    outs = [DeviceColumn(1 << (log_n + 1)) for _ in range(n_cols)]
    ti = te = 0.0
    for it in range(iters):
        sync()
        t0 = time.perf_counter()
        be.interpolate_columns_into(evals, coeffs, tree)
        sync()
        t1 = time.perf_counter()
        be.evaluate_polynomials_into(coeffs, 1, tree, outs)
        sync()
        t2 = time.perf_counter()
        if it >= 2:
            ti += t1 - t0
            te += t2 - t1
    k = max(1, iters - 2)
    el_i = n_cols * (1 << log_n) * log_n
    el_e = n_cols * (1 << (log_n + 1)) * log_n
    print(f"interpolate {ti / k * 1e3:.3f} ms ({el_i / (ti / k) / 1e12:.3f} T element-layers/s); "
          f"evaluate {te / k * 1e3:.3f} ms ({el_e / (te / k) / 1e12:.3f} T element-layers/s)")


if __name__ == "__main__":
    main()
