"""The oracle's QuotientOps / AccumulationOps restatement against the
reference's own structural tests (CPU only).

- prover/pcs/quotient_ops.rs tests (test_quotients_are_low_degree): the FRI
  quotient of a polynomial's evaluation by its value at a circle point of the
  secure field is a polynomial of lower degree, so interpolating the quotient
  leaves the top coefficients zero.
- prover/backend/cpu/accumulation.rs (test_lift_and_accumulate): the lifted sum
  equals the sum of each column read at the lifted index.
- generate_secure_powers: felt^k by repeated multiplication.
"""
import numpy as np

P = (1 << 31) - 1


def qadd(a, b):
    return tuple((int(x) + int(y)) % P for x, y in zip(a, b))


def qsub(a, b):
    return tuple((int(x) - int(y)) % P for x, y in zip(a, b))


def random_secure_point(oracle, rng):
    # ((1 - t^2) / (1 + t^2), 2t / (1 + t^2)) for a random QM31 t (core/circle.rs:169-181)
    t = tuple(int(x) for x in rng.integers(0, P, 4))
    t2 = oracle.qm31_mul(t, t)
    inv1 = oracle.qm31_inv(qadd(t2, (1, 0, 0, 0)))
    x = oracle.qm31_mul(qsub((1, 0, 0, 0), t2), inv1)
    y = oracle.qm31_mul(qadd(t, t), inv1)
    return np.array(x + y, np.uint32)


def test_quotient_of_sampled_polynomial_is_low_degree(oracle):
    rng = np.random.default_rng(77)
    log_n, log_blowup = 6, 2
    L = log_n + log_blowup
    init, lg = oracle.canonic_half_coset_root(L + 1)
    tw, itw = oracle.precompute_twiddles(init, lg)
    polys = [rng.integers(0, P, 1 << log_n, dtype=np.uint32) for _ in range(3)]
    evals = [oracle.evaluate(c, L, tw) for c in polys]
    z = random_secure_point(oracle, rng)
    alpha = rng.integers(0, P, 4, dtype=np.uint32)
    terms, a_pow = [], np.array([1, 0, 0, 0], np.uint32)
    for k, c in enumerate(polys):
        terms.append((k, oracle.eval_at_secure_point(c, z), a_pow))
        a_pow = np.array(oracle.qm31_mul(a_pow, alpha), np.uint32)
    num, first = oracle.accumulate_numerators(evals, L, z, terms)
    quot = oracle.compute_quotients_and_combine([(z, num, first)], L)
    for coord in quot:
        coeffs = oracle.interpolate(coord, itw)
        assert (coeffs[1 << log_n:] == 0).all()
        assert coeffs[: 1 << log_n].any()
    # a wrong sampled value breaks it
    bad = [(0, qadd(terms[0][1], (1, 0, 0, 0)), terms[0][2])] + terms[1:]
    num, first = oracle.accumulate_numerators(evals, L, z, bad)
    quot = oracle.compute_quotients_and_combine([(z, num, first)], L)
    assert any(oracle.interpolate(c, itw)[1 << log_n:].any() for c in quot)


def test_lift_and_accumulate_is_the_sum_of_lifts(oracle):
    rng = np.random.default_rng(78)
    logs = [4, 5, 8]
    cols = [[rng.integers(0, P, 1 << l, dtype=np.uint32) for _ in range(4)] for l in logs]
    out = oracle.lift_and_accumulate(cols)
    L = logs[-1]
    i = np.arange(1 << L, dtype=np.int64)
    for c in range(4):
        ref = np.zeros(1 << L, np.int64)
        for col, l in zip(cols, logs):
            r = L - l
            j = i if r == 0 else ((i >> (r + 1)) << 1) + (i & 1)
            ref = (ref + col[c][j].astype(np.int64)) % P
        assert (out[c].astype(np.int64) == ref).all()


def test_generate_secure_powers(oracle):
    felt = (12345, 678, 9, 1011)
    pw = oracle.generate_secure_powers(felt, 9)
    acc = (1, 0, 0, 0)
    for k in range(9):
        assert tuple(int(x) for x in pw[k]) == acc
        acc = oracle.qm31_mul(acc, felt)
