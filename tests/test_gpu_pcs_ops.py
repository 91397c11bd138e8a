"""The trait methods beside commit and FRI (QuotientOps, AccumulationOps,
PolyOps::eval_at_point, GrindOps, ColumnOps<SecureField>) through the C ABI,
bit-exact against the oracle on seeded inputs, including the reference's edge
cases: P-valued words, small sizes, chunked launches (more than 256 terms,
more than 8 sample points) and lifts of several sizes."""
import numpy as np
import pytest

from stwo_b200 import B200Backend, DeviceBuffer, DeviceColumn, SecureColumn

pytestmark = pytest.mark.gpu
P = (1 << 31) - 1


@pytest.fixture(scope="module")
def be():
    return B200Backend()


def rq(rng):
    return rng.integers(0, P, 4, dtype=np.uint32)


def rpoint(rng):
    return rng.integers(0, P, 8, dtype=np.uint32)


def check_secure(got: SecureColumn, ref):
    for g, r in zip(got.to_host(), ref):
        assert (g == r).all()


@pytest.mark.parametrize("log_n,n_cols,n_terms", [(0, 3, 2), (3, 5, 7), (10, 20, 40), (14, 6, 300), (18, 100, 108)])
def test_accumulate_numerators(be, oracle, log_n, n_cols, n_terms):
    rng = np.random.default_rng(1000 + log_n)
    cols = [rng.integers(0, P, 1 << log_n, dtype=np.uint32) for _ in range(n_cols)]
    cols[0][: min(4, cols[0].size)] = P  # words equal to P
    dev = [DeviceColumn.from_host(c) for c in cols]
    batches = []
    for _ in range(2):
        terms = [(int(rng.integers(0, n_cols)), rq(rng), rq(rng)) for _ in range(n_terms)]
        batches.append((rpoint(rng), terms))
    got = be.accumulate_numerators(dev, batches)
    for (point, terms), (col, first) in zip(batches, got):
        ref, ref_first = oracle.accumulate_numerators(cols, log_n, point, terms)
        check_secure(col, ref)
        assert (first == ref_first).all()


@pytest.mark.parametrize("lifting,logs", [(5, [5]), (8, [3, 5, 8]), (12, [12, 9, 4, 12, 7, 10, 11, 12, 6, 8]),
                                          (16, [16, 13])])
def test_compute_quotients_and_combine(be, oracle, lifting, logs):
    rng = np.random.default_rng(2000 + lifting)
    accs, dev_accs = [], []
    for l in logs:
        part = [rng.integers(0, P, 1 << l, dtype=np.uint32) for _ in range(4)]
        point, first = rpoint(rng), rq(rng)
        accs.append((point, part, first))
        dev_accs.append((point, SecureColumn.from_host(part), first))
    got = be.compute_quotients_and_combine(dev_accs, lifting)
    check_secure(got, oracle.compute_quotients_and_combine(accs, lifting))


def test_fri_quotients_chain_matches_oracle(be, oracle):
    # compute_fri_quotients (prover/pcs/quotient_ops.rs:134-233) over two
    # column sizes and two sample points: numerators per size, lifted and
    # summed per point, then combined on the lifting domain.
    rng = np.random.default_rng(3000)
    L = 11
    sizes = {9: 7, 11: 5}
    points = [rpoint(rng), rpoint(rng)]
    per_point = {0: [], 1: []}
    per_point_ref = {0: [], 1: []}
    for l in sorted(sizes):
        cols = [rng.integers(0, P, 1 << l, dtype=np.uint32) for _ in range(sizes[l])]
        dev = [DeviceColumn.from_host(c) for c in cols]
        batches = [(points[z], [(k, rq(rng), rq(rng)) for k in range(sizes[l])]) for z in range(2)]
        got = be.accumulate_numerators(dev, batches)
        for z, (point, terms) in enumerate(batches):
            per_point[z].append(got[z])
            per_point_ref[z].append(oracle.accumulate_numerators(cols, l, point, terms))
    accs, accs_ref = [], []
    for z in range(2):
        lifted = be.lift_and_accumulate([c for c, _ in per_point[z]])
        firsts = [f for _, f in per_point[z]]
        first = np.array([sum(int(f[k]) for f in firsts) % P for k in range(4)], np.uint32)
        accs.append((points[z], lifted, first))
        lifted_ref = oracle.lift_and_accumulate([c for c, _ in per_point_ref[z]])
        firsts_ref = [f for _, f in per_point_ref[z]]
        assert all((a == b).all() for a, b in zip(firsts, firsts_ref))
        accs_ref.append((points[z], lifted_ref, first))
    check_secure(be.compute_quotients_and_combine(accs, L), oracle.compute_quotients_and_combine(accs_ref, L))


@pytest.mark.parametrize("logs", [[4], [4, 6, 9], [1, 2, 5, 20], [10, 11, 12, 13, 14, 15, 16]])
def test_lift_and_accumulate(be, oracle, logs):
    rng = np.random.default_rng(4000 + sum(logs))
    cols = [[rng.integers(0, P, 1 << l, dtype=np.uint32) for _ in range(4)] for l in logs]
    cols[0][0][0] = P  # the first column is taken as it is (P stays P where nothing is added)
    dev = [SecureColumn.from_host(c) for c in cols]
    got = be.lift_and_accumulate(dev)
    check_secure(got, oracle.lift_and_accumulate(cols))
    # in place into the last column, as the trait consumes it
    be.lift_and_accumulate(dev, out=dev[-1])
    check_secure(dev[-1], oracle.lift_and_accumulate(cols))


@pytest.mark.parametrize("n", [1, 5, 1 << 16])
def test_accumulate(be, oracle, n):
    rng = np.random.default_rng(5000 + n)
    a = [rng.integers(0, P, n, dtype=np.uint32) for _ in range(4)]
    b = [rng.integers(0, P, n, dtype=np.uint32) for _ in range(4)]
    a[0][0], b[0][0] = P, P
    a[1][0], b[1][0] = P, 0
    da, db = SecureColumn.from_host(a), SecureColumn.from_host(b)
    be.accumulate(da, db)
    check_secure(da, oracle.accumulate(a, b))


@pytest.mark.parametrize("n", [0, 1, 17, 1000])
def test_generate_secure_powers(be, oracle, n):
    felt = np.array([123456789, 987654321, 5, 2147483646], np.uint32)
    assert (be.generate_secure_powers(felt, n) == oracle.generate_secure_powers(felt, n)).all()


# 13..24 run the bucketed form (1024-index buckets, 8 per warp), the others
# the chunked one.
@pytest.mark.parametrize("log_n", [0, 1, 2, 5, 8, 9, 10, 11, 12, 13, 16, 20, 21, 24])
def test_eval_at_point(be, oracle, log_n):
    rng = np.random.default_rng(6000 + log_n)
    polys = [rng.integers(0, P, 1 << log_n, dtype=np.uint32) for _ in range(3)]
    polys[1][0] = P
    polys[0][rng.integers(0, 1 << log_n, 1 + (1 << log_n) // 64)] = P  # words equal to P count as 0
    point = rpoint(rng)
    dev = [DeviceColumn.from_host(c) for c in polys]
    got = be.batch_eval_at_point(dev, point)
    for k, c in enumerate(polys):
        ref = oracle.eval_at_secure_point(c, point)
        assert (got[k] == ref).all(), k
    assert (be.eval_at_point(dev[2], point) == oracle.eval_at_secure_point(polys[2], point)).all()


@pytest.mark.parametrize("log_n", [6, 14])
def test_batch_eval_at_point_many_polys(be, oracle, log_n):
    rng = np.random.default_rng(6100 + log_n)
    polys = [rng.integers(0, P, 1 << log_n, dtype=np.uint32) for _ in range(1030)]  # two launches
    point = rpoint(rng)
    got = be.batch_eval_at_point([DeviceColumn.from_host(c) for c in polys], point)
    for k in (0, 511, 1023, 1024, 1029):
        assert (got[k] == oracle.eval_at_secure_point(polys[k], point)).all()


@pytest.mark.parametrize("bits,m31", [(0, False), (1, False), (8, True), (12, False), (18, False), (18, True)])
def test_grind(be, oracle, bits, m31):
    rng = np.random.default_rng(7000 + bits)
    ch = oracle.Channel(m31)
    ch.mix_u32s(rng.integers(0, P, 8, dtype=np.uint32))
    nonce = be.grind(ch.digest, bits, m31)
    assert nonce == ch.grind(bits)
    assert ch.verify_pow(bits, nonce)


@pytest.mark.parametrize("log_n", [0, 1, 4, 11, 17])
def test_bit_reverse_secure(be, oracle, log_n):
    rng = np.random.default_rng(8000 + log_n)
    coords = [rng.integers(0, P, 1 << log_n, dtype=np.uint32) for _ in range(4)]
    sc = SecureColumn.from_host(coords)
    be.bit_reverse_secure_column(sc)
    check_secure(sc, [oracle.bit_reverse(c) for c in coords])
    aos = np.stack(coords, axis=1).reshape(-1)
    buf = DeviceBuffer(aos.nbytes)
    buf.upload(aos)
    be.bit_reverse_secure_field(buf, log_n)
    ref = np.stack([oracle.bit_reverse(c) for c in coords], axis=1).reshape(-1)
    assert (buf.download(np.uint32, aos.size) == ref).all()
