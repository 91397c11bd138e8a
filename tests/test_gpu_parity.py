"""GPU parity: every B200 kernel against the CPU oracle, bit-exact, through
the C ABI.  Sizes cover the reference's edge cases: tiny domains (log 1-5,
where SimdBackend falls back to CPU code), log 16/17 (the SIMD transpose
boundary), columns < 16, = 16 and 17 (Blake2s block boundary), uneven size
groups and P-valued words."""
import numpy as np
import pytest

from stwo_b200 import B200Backend, DeviceColumn, SecureColumn, layer_to_host

pytestmark = pytest.mark.gpu
P = (1 << 31) - 1


@pytest.fixture(scope="module")
def be():
    return B200Backend()


def rng(seed):
    return np.random.default_rng(seed)


def rand_col(r, log_n):
    return r.integers(0, P, 1 << log_n, dtype=np.uint32)


@pytest.mark.parametrize("log_size", [0, 1, 2, 3, 5, 10, 16, 21])
def test_twiddles(be, oracle, log_size):
    init = 1 << (31 - (log_size + 2))
    tree = be.precompute_twiddles(init, log_size)
    tw, itw = oracle.precompute_twiddles(init, log_size)
    assert (tree.twiddles.to_host() == tw).all()
    assert (tree.itwiddles.to_host() == itw).all()


@pytest.mark.parametrize("log_n", [1, 2, 5, 10, 17, 20])
def test_bit_reverse(be, oracle, log_n):
    v = rand_col(rng(log_n), log_n)
    c = DeviceColumn.from_host(v)
    be.bit_reverse_column(c)
    assert (c.to_host() == oracle.bit_reverse(v)).all()


@pytest.mark.parametrize("in_place", [False, True])
def test_bit_reverse_columns(be, oracle, in_place):
    # a batch with runs of equal sizes, including log 0 and a run longer than
    # one launch's column table
    logs = [0, 3, 3, 7, 7, 7, 12] + [5] * 300 + [16]
    r = rng(77)
    vals = [rand_col(r, l) for l in logs]
    srcs = [DeviceColumn.from_host(v) for v in vals]
    dsts = None if in_place else [DeviceColumn(1 << l) for l in logs]
    be.bit_reverse_columns(srcs, dsts)
    for v, c in zip(vals, srcs if in_place else dsts):
        assert (c.to_host() == oracle.bit_reverse(v)).all()
    if not in_place:  # sources untouched
        for v, c in zip(vals, srcs):
            assert (c.to_host() == v).all()


LOGS = [1, 2, 3, 4, 5, 6, 8, 11, 12, 13, 16, 17, 20, 22]


@pytest.fixture(scope="module")
def big_tree(be, oracle):
    init, lg = oracle.canonic_half_coset_root(25)
    tw, itw = oracle.precompute_twiddles(init, lg)
    return be.precompute_twiddles(init, lg), tw, itw


@pytest.mark.parametrize("log_n", LOGS)
def test_interpolate(be, oracle, big_tree, log_n):
    tree, tw, itw = big_tree
    vals = [rand_col(rng(1000 + log_n + k), log_n) for k in range(3)]
    cols = [DeviceColumn.from_host(v) for v in vals]
    be.interpolate_columns(cols, tree)
    for v, c in zip(vals, cols):
        assert (c.to_host() == oracle.interpolate(v, itw)).all()


@pytest.mark.parametrize("log_n", [1, 2, 3, 9, 10, 11, 12, 16, 17, 20, 22])
@pytest.mark.parametrize("in_place", [False, True])
def test_interpolate_natural(be, oracle, big_tree, log_n, in_place):
    # natural-order evaluations: bit reversal + interpolation in one call (the
    # bit reversal fused into the first pass from log 3 up, out of place);
    # 11 columns leave a partial group of 8; P-valued words included
    tree, tw, itw = big_tree
    r = rng(3000 + log_n)
    vals = [rand_col(r, log_n) for _ in range(11 if log_n <= 17 else 2)]
    vals[0][:: max(1, len(vals[0]) // 7)] = P
    srcs = [DeviceColumn.from_host(v) for v in vals]
    dsts = srcs if in_place else [DeviceColumn(1 << log_n) for _ in vals]
    be.interpolate_natural_into(srcs, dsts, tree)
    for v, d in zip(vals, dsts):
        assert (d.to_host() == oracle.interpolate(oracle.bit_reverse(v), itw)).all()
    if not in_place:
        for v, c in zip(vals, srcs):
            assert (c.to_host() == v).all()


def test_interpolate_natural_mixed_sizes_and_plans(be, oracle, big_tree):
    # uneven sizes in one call, under the default plans and with log 12 as
    # 6 + 6 layers (a tile first pass instead of the single 12-layer one)
    from stwo_b200 import fft_get_plan, fft_set_plan
    tree, tw, itw = big_tree
    r = rng(31)
    logs = [12, 3, 14, 12, 10, 1, 14, 18, 12]
    vals = [rand_col(r, l) for l in logs]
    old = fft_get_plan(12)
    try:
        for plan in ([], [6, 6]):
            fft_set_plan(12, plan)
            srcs = [DeviceColumn.from_host(v) for v in vals]
            dsts = [DeviceColumn(1 << l) for l in logs]
            be.interpolate_natural_into(srcs, dsts, tree)
            for v, d in zip(vals, dsts):
                assert (d.to_host() == oracle.interpolate(oracle.bit_reverse(v), itw)).all(), (plan, v.size)
    finally:
        fft_set_plan(12, old)


@pytest.mark.parametrize("log_n", LOGS)
@pytest.mark.parametrize("log_blowup", [0, 1, 2])
def test_evaluate(be, oracle, big_tree, log_n, log_blowup):
    tree, tw, itw = big_tree
    coeffs = [rand_col(rng(2000 + log_n), log_n)]
    outs = be.evaluate_polynomials([DeviceColumn.from_host(coeffs[0])], log_blowup, tree)
    ref = oracle.evaluate(coeffs[0], log_n + log_blowup, tw)
    assert (outs[0].to_host() == ref).all()


def test_uneven_batch_roundtrip(be, oracle, big_tree):
    tree, tw, itw = big_tree
    r = rng(7)
    logs = [int(x) for x in r.integers(3, 15, 40)]
    vals = [rand_col(r, l) for l in logs]
    cols = [DeviceColumn.from_host(v) for v in vals]
    be.interpolate_columns(cols, tree)
    evs = be.evaluate_polynomials(cols, 2, tree)
    for v, c, e, l in zip(vals, cols, evs, logs):
        co = oracle.interpolate(v, itw)
        assert (c.to_host() == co).all()
        assert (e.to_host() == oracle.evaluate(co, l + 2, tw)).all()


@pytest.mark.parametrize("log_n,log_blowup", [(1, 1), (3, 1), (8, 2), (16, 1), (20, 0), (20, 1), (20, 2), (21, 1),
                                               (21, 2)])
@pytest.mark.parametrize("in_place", [False, True])
def test_interpolate_evaluate(be, oracle, big_tree, log_n, log_blowup, in_place):
    # interpolate_columns + evaluate_polynomials in one call: at logs 20 and 21
    # with blowup 1 the interpolation's last pass and the evaluation's first
    # are one kernel (separate passes at blowup 2).  Words equal to P included.
    tree, tw, itw = big_tree
    r = rng(3000 + log_n)
    vals = [rand_col(r, log_n) for _ in range(3)]
    vals[1][::5] = P
    srcs = [DeviceColumn.from_host(v) for v in vals]
    coeffs = srcs if in_place else [DeviceColumn(1 << log_n) for _ in vals]
    outs = [DeviceColumn(1 << (log_n + log_blowup)) for _ in vals]
    be.interpolate_evaluate_into(None if in_place else srcs, coeffs, log_blowup, tree, outs)
    for k, v in enumerate(vals):
        co = oracle.interpolate(v, itw)
        assert (coeffs[k].to_host() == co).all(), k
        assert (outs[k].to_host() == oracle.evaluate(co, log_n + log_blowup, tw)).all(), k
        if not in_place:
            assert (srcs[k].to_host() == v).all()


@pytest.mark.parametrize("log_n,plan", [(13, [3, 10]), (15, [5, 10]), (16, [6, 10])])
def test_strided_pass_runtime_layer_offset(be, oracle, big_tree, log_n, plan):
    # Splits ending in a 10-layer pass that starts at layer 3..9: the strided
    # warp kernel with the layer offset read at run time (the autotuner can
    # pick these), for the interpolation and for blowup-1 and -2 evaluations.
    from stwo_b200 import fft_get_plan, fft_set_plan
    tree, tw, itw = big_tree
    old = fft_get_plan(log_n)
    fft_set_plan(log_n, plan)
    try:
        r = rng(3300 + log_n)
        vals = [rand_col(r, log_n) for _ in range(3)]
        vals[2][::9] = P
        cols = [DeviceColumn.from_host(v) for v in vals]
        be.interpolate_columns(cols, tree)
        for blowup in (1, 2):
            evs = be.evaluate_polynomials(cols, blowup, tree)
            for k, v in enumerate(vals):
                co = oracle.interpolate(v, itw)
                assert (cols[k].to_host() == co).all(), k
                assert (evs[k].to_host() == oracle.evaluate(co, log_n + blowup, tw)).all(), (k, blowup)
    finally:
        fft_set_plan(log_n, old)


def test_interpolate_evaluate_many_columns(be, oracle, big_tree):
    # 260 columns of log 20 in one call: the fused kernel launches per 256
    # columns; columns on both sides of the boundary against the oracle.
    tree, tw, itw = big_tree
    r = rng(3200)
    base = [rand_col(r, 20) for _ in range(4)]
    picks = {0: 0, 255: 1, 256: 2, 259: 3}
    srcs = [DeviceColumn.from_host(base[picks.get(k, k % 4)]) for k in range(260)]
    coeffs = [DeviceColumn(1 << 20) for _ in range(260)]
    outs = [DeviceColumn(1 << 21) for _ in range(260)]
    be.interpolate_evaluate_into(srcs, coeffs, 1, tree, outs)
    for k, b in picks.items():
        co = oracle.interpolate(base[b], itw)
        assert (coeffs[k].to_host() == co).all(), k
        assert (outs[k].to_host() == oracle.evaluate(co, 21, tw)).all(), k


def candidate_splits(n):
    """The pass splits the committer's autotuner times for an n-layer FFT
    (every one of them can end up in the plan table)."""
    c = [[n]] if n <= 12 else []
    c += [[a, n - a] for a in range(3, min(12, n - 1) + 1) if 1 <= n - a <= 12]
    if n >= 15:
        for a in range(max(3, n // 3 - 1), min(12, n // 3 + 1) + 1):
            for b in range(max(1, (n - a) // 2 - 1), min(12, (n - a) // 2 + 1) + 1):
                if 1 <= n - a - b <= 12:
                    c.append([a, b, n - a - b])
    return c


@pytest.mark.parametrize("log_n,n_cols", [(13, 9), (14, 9), (16, 9), (19, 5), (22, 3)])
def test_every_candidate_split(be, oracle, big_tree, log_n, n_cols):
    # Whatever split the autotuner keeps, each pass shape it implies (warp,
    # group or tile kernels, contiguous and strided, every layer offset) gives
    # the oracle's coefficients and blowup-1 and -2 evaluations; 9 columns
    # leave a partial column group (fewer columns at logs 19 and 22).
    from stwo_b200 import fft_get_plan, fft_set_plan
    tree, tw, itw = big_tree
    r = rng(3600 + log_n)
    vals = [rand_col(r, log_n) for _ in range(n_cols)]
    vals[n_cols // 2][::7] = P
    co = [oracle.interpolate(v, itw) for v in vals]
    ev = {b: [oracle.evaluate(c, log_n + b, tw) for c in co] for b in (1, 2)}
    old = fft_get_plan(log_n)
    try:
        for plan in candidate_splits(log_n):
            fft_set_plan(log_n, plan)
            cols = [DeviceColumn.from_host(v) for v in vals]
            for b in (1, 2):
                outs = [DeviceColumn(1 << (log_n + b)) for _ in vals]
                be.interpolate_evaluate_into(cols if b == 1 else None, [DeviceColumn(1 << log_n) for _ in vals]
                                             if b == 1 else cols, b, tree, outs)
                for k in range(len(vals)):
                    assert (outs[k].to_host() == ev[b][k]).all(), (plan, b, k)
            for k in range(len(vals)):
                assert (cols[k].to_host() == co[k]).all(), (plan, k)
    finally:
        fft_set_plan(log_n, old)


@pytest.mark.parametrize("log_n,plan", [(13, [7, 6]), (14, [6, 8]), (15, [9, 6]), (16, [6, 10]), (12, [8, 4]),
                                        (11, [9, 2]), (10, [6, 4])])
def test_short_contiguous_passes(be, oracle, big_tree, log_n, plan):
    # First (inverse) / last (forward) passes of 6..9 layers on the contiguous
    # warp kernel, 2^(10 - T) tiles per 1024-word warp tile, for natural- and
    # bit-reversed-order interpolation and evaluations at blowups 0..2.
    from stwo_b200 import fft_get_plan, fft_set_plan
    tree, tw, itw = big_tree
    old = fft_get_plan(log_n)
    fft_set_plan(log_n, plan)
    try:
        r = rng(3500 + log_n + plan[0])
        vals = [rand_col(r, log_n) for _ in range(9)]
        vals[2][::3] = P
        cols = [DeviceColumn.from_host(v) for v in vals]
        nat = [DeviceColumn(1 << log_n) for _ in vals]
        be.interpolate_natural_into([DeviceColumn.from_host(oracle.bit_reverse(v)) for v in vals], nat, tree)
        be.interpolate_columns(cols, tree)
        for blowup in (0, 1, 2):
            evs = be.evaluate_polynomials(cols, blowup, tree)
            for k, v in enumerate(vals):
                co = oracle.interpolate(v, itw)
                if blowup == 0:
                    assert (cols[k].to_host() == co).all(), k
                    assert (nat[k].to_host() == co).all(), k
                assert (evs[k].to_host() == oracle.evaluate(co, log_n + blowup, tw)).all(), (k, blowup)
    finally:
        fft_set_plan(log_n, old)


@pytest.mark.parametrize("log_n,plan", [(16, [10, 6]), (17, [10, 7]), (18, [10, 8]), (19, [10, 9]), (19, [11, 8]),
                                        (15, [7, 8]), (13, [7, 6]), (14, [5, 9])])
def test_short_strided_passes(be, oracle, big_tree, log_n, plan):
    # Second passes of 6..9 layers: the warp kernel that puts 2^(10 - T) tiles
    # of the pass side by side in one block (layer offsets 10 and 11 fixed at
    # compile time, others read at run time), for the interpolation and for
    # evaluations at blowups 0..2 (the duplicated coefficients masked).
    from stwo_b200 import fft_get_plan, fft_set_plan
    tree, tw, itw = big_tree
    old = fft_get_plan(log_n)
    fft_set_plan(log_n, plan)
    try:
        r = rng(3400 + log_n + plan[0])
        vals = [rand_col(r, log_n) for _ in range(3)]
        vals[1][::3] = P
        cols = [DeviceColumn.from_host(v) for v in vals]
        be.interpolate_columns(cols, tree)
        for blowup in (0, 1, 2):
            evs = be.evaluate_polynomials(cols, blowup, tree)
            for k, v in enumerate(vals):
                co = oracle.interpolate(v, itw)
                if blowup == 0:
                    assert (cols[k].to_host() == co).all(), k
                assert (evs[k].to_host() == oracle.evaluate(co, log_n + blowup, tw)).all(), (k, blowup)
    finally:
        fft_set_plan(log_n, old)


@pytest.mark.parametrize("log_n,plan,n_cols", [(22, [12, 10], 15), (21, [11, 10], 27)])
def test_group_passes_loop_over_columns(be, oracle, big_tree, log_n, plan, n_cols):
    # Enough columns that the 11- and 12-layer contiguous passes give each
    # warp group several columns of one tile position (the interpolation's
    # first pass and the blowup-2 evaluation's last), with a ragged last
    # group; three distinct columns repeated, checked at every position.
    from stwo_b200 import fft_get_plan, fft_set_plan
    tree, tw, itw = big_tree
    old = fft_get_plan(log_n)
    fft_set_plan(log_n, plan)
    try:
        r = rng(3300 + log_n)
        base = [rand_col(r, log_n) for _ in range(3)]
        base[1][::5] = P
        srcs = [DeviceColumn.from_host(base[k % 3]) for k in range(n_cols)]
        coeffs = [DeviceColumn(1 << log_n) for _ in range(n_cols)]
        outs = [DeviceColumn(1 << (log_n + 2)) for _ in range(n_cols)]
        be.interpolate_evaluate_into(srcs, coeffs, 2, tree, outs)
        ref = []
        for b in base:
            co = oracle.interpolate(b, itw)
            ref.append((co, oracle.evaluate(co, log_n + 2, tw)))
        for k in range(n_cols):
            assert (coeffs[k].to_host() == ref[k % 3][0]).all(), k
            assert (outs[k].to_host() == ref[k % 3][1]).all(), k
    finally:
        fft_set_plan(log_n, old)


@pytest.mark.parametrize("log_blowup", [1, 2])
def test_interpolate_evaluate_layer12_plan(be, oracle, big_tree, log_blowup):
    # Log 22 under the split [12, 10] (the uneven commit's autotuned plan):
    # the 10-layer strided passes start at layer 12, fused in the one call at
    # blowup 1 and separate in the two trait calls (and at blowup 2).
    from stwo_b200 import fft_get_plan, fft_set_plan
    tree, tw, itw = big_tree
    old = fft_get_plan(22)
    fft_set_plan(22, [12, 10])
    try:
        r = rng(3100 + log_blowup)
        vals = [rand_col(r, 22) for _ in range(2)]
        vals[0][::7] = P
        srcs = [DeviceColumn.from_host(v) for v in vals]
        coeffs = [DeviceColumn(1 << 22) for _ in vals]
        outs = [DeviceColumn(1 << (22 + log_blowup)) for _ in vals]
        be.interpolate_evaluate_into(srcs, coeffs, log_blowup, tree, outs)
        c2 = [DeviceColumn(1 << 22) for _ in vals]
        be.interpolate_columns_into(srcs, c2, tree)
        o2 = be.evaluate_polynomials(c2, log_blowup, tree)
        for k, v in enumerate(vals):
            co = oracle.interpolate(v, itw)
            ev = oracle.evaluate(co, 22 + log_blowup, tw)
            assert (coeffs[k].to_host() == co).all() and (c2[k].to_host() == co).all(), k
            assert (outs[k].to_host() == ev).all() and (o2[k].to_host() == ev).all(), k
    finally:
        fft_set_plan(22, old)


def test_p_valued_inputs(be, oracle, big_tree):
    # Words equal to P (the redundant zero) propagate exactly like SimdBackend.
    tree, tw, itw = big_tree
    for log_n in [3, 6, 12, 14]:
        v = rand_col(rng(log_n), log_n)
        v[::3] = P
        v[1::7] = 0
        c = DeviceColumn.from_host(v)
        be.interpolate_columns([c], tree)
        assert (c.to_host() == oracle.interpolate(v, itw)).all()
        e = be.evaluate_polynomials([DeviceColumn.from_host(v)], 1, tree)[0]
        assert (e.to_host() == oracle.evaluate(v, log_n + 1, tw)).all()


@pytest.mark.parametrize("logs,L", [
    ([4, 4, 4], 4),
    ([2, 3, 4], 4),
    ([5] * 16, 5),
    ([5] * 17, 5),
    ([3, 7, 7, 1, 9, 9, 9, 2] + [6] * 20, 11),
    ([10] * 33, 12),
])
@pytest.mark.parametrize("m31", [False, True])
def test_merkle_layers(be, oracle, logs, L, m31):
    r = rng(sum(logs) + L)
    vals = [rand_col(r, l) for l in logs]
    cols = [DeviceColumn.from_host(v) for v in vals]
    layers = be.build_merkle_layers(cols, L, m31)
    ref = oracle.merkle_build_layers(vals, L, m31)
    for k in range(L + 1):
        assert (layer_to_host(layers[k]) == ref[k]).all(), k


@pytest.mark.parametrize("logs,L", [([19, 17], 19), ([20, 22], 22)])
@pytest.mark.parametrize("m31", [False, True])
def test_merkle_layers_wide(be, oracle, logs, L, m31):
    # lifting sizes >= 19 take the three-levels-per-thread node kernel (twice at 22)
    test_merkle_layers(be, oracle, logs, L, m31)


def test_merkle_empty(be, oracle):
    layers = be.build_merkle_layers([], 0)
    assert (layer_to_host(layers[0]) == oracle.merkle_build_layers([], 0)[0]).all()


def test_merkle_many_columns_chunked(be, oracle):
    # More columns than one leaf launch holds: the chaining state is carried.
    r = rng(99)
    logs = [4] * 1100 + [6] * 30
    vals = [rand_col(r, l) for l in logs]
    cols = [DeviceColumn.from_host(v) for v in vals]
    layers = be.build_merkle_layers(cols, 7)
    ref = oracle.merkle_build_layers(vals, 7)
    assert (layer_to_host(layers[0]) == ref[0]).all()
    assert (layer_to_host(layers[7]) == ref[7]).all()


STAGED_LEAF_CASES = [
    # (log sizes, lifting log size): the leaves run in stages, one per run of
    # 16-column compression groups of one largest log size, the chaining
    # values lifted between stages
    (sorted(int(x) for x in np.random.default_rng(7).integers(1, 13, 200)), 12),  # mixed groups, many stages
    (sorted(int(x) for x in np.random.default_rng(8).integers(1, 11, 90)), 13),   # last group alone at L > max
    ([3] * 1200 + [6] * 40, 6),   # 75 groups of one size: two launches, the second in place
    ([5] * 1100, 5),              # 69 groups at L: the first launch leaves its chaining values for the second
    ([1] * 16 + [2] * 16 + [9], 9),  # one group per stage, the last one partial
]


@pytest.mark.parametrize("logs,L", STAGED_LEAF_CASES)
@pytest.mark.parametrize("m31", [False, True])
def test_lifted_leaves_stages(be, oracle, logs, L, m31):
    r = rng(len(logs) + L)
    vals = [rand_col(r, l) for l in logs]
    cols = [DeviceColumn.from_host(v) for v in vals]
    ref = oracle.merkle_build_layers(vals, L, m31)
    # with the tree's layer buffers as the stages' chaining values
    layers = be.build_merkle_layers(cols, L, m31)
    for k in range(L + 1):
        assert (layer_to_host(layers[k]) == ref[k]).all(), k
    # leaves alone: the chaining values packed in a temporary buffer
    assert (layer_to_host(be.build_leaves(cols, L, m31)) == ref[L]).all()
    # leaves into caller-owned layers (build_leaves_layers), then the nodes
    from stwo_b200 import DeviceBuffer
    own = [DeviceBuffer(32 << k) for k in range(L + 1)]
    assert (layer_to_host(be.build_leaves_layers(cols, L, own, m31)) == ref[L]).all()
    be.build_nodes(own, m31)
    for k in range(L + 1):
        assert (layer_to_host(own[k]) == ref[k]).all(), k


def test_lifted_leaves_reject_bad_columns(be):
    # build_leaves and build_leaves_layers take columns already sorted by
    # length, none larger than the lifting size
    from stwo_b200 import DeviceBuffer
    from stwo_b200.ffi import B200Error
    r = rng(11)
    cols = [DeviceColumn.from_host(rand_col(r, l)) for l in (5, 3)]
    with pytest.raises(B200Error, match="sorted"):
        be.build_leaves(cols, 6)
    with pytest.raises(B200Error, match="exceeds"):
        be.build_leaves(cols[::-1], 4)
    with pytest.raises(B200Error, match="sorted"):
        be.build_leaves_layers(cols, 6, [DeviceBuffer(32 << k) for k in range(7)])


def test_build_leaves_and_next_layer(be, oracle):
    r = rng(5)
    vals = [rand_col(r, l) for l in [3, 5, 5, 8]]
    cols = [DeviceColumn.from_host(v) for v in vals]
    leaves = be.build_leaves(cols, 9)
    ref = oracle.merkle_build_leaves(vals, 9)
    assert (layer_to_host(leaves) == ref).all()
    nxt = be.build_next_layer(leaves)
    assert (layer_to_host(nxt) == oracle.merkle_next_layer(ref)).all()


@pytest.mark.parametrize("with_prev", [False, True])
@pytest.mark.parametrize("n_cols", [0, 1, 16, 17])
def test_commit_on_layer(be, oracle, with_prev, n_cols):
    r = rng(n_cols * 2 + with_prev)
    log_size = 6
    vals = [rand_col(r, log_size) for _ in range(n_cols)]
    prev_host = r.integers(0, 256, (2 << log_size, 32), dtype=np.uint8) if with_prev else None
    prev = None
    if with_prev:
        from stwo_b200 import DeviceBuffer
        prev = DeviceBuffer(prev_host.nbytes)
        prev.upload(prev_host)
    out = be.commit_on_layer(log_size, prev, [DeviceColumn.from_host(v) for v in vals])
    ref = oracle.commit_on_layer(log_size, prev_host, vals)
    assert (layer_to_host(out) == ref).all()


def test_mixed_degree_commit_matches_oracle(be, oracle):
    r = rng(11)
    logs = [6, 4, 6, 2, 5]
    vals = [rand_col(r, l) for l in logs]
    ref = oracle.mixed_degree_commit(vals)
    order = sorted(range(len(vals)), key=lambda i: -logs[i])
    prev = None
    for log_size in range(6, -1, -1):
        cs = [DeviceColumn.from_host(vals[i]) for i in order if logs[i] == log_size]
        prev = be.commit_on_layer(log_size, prev, cs)
        assert (layer_to_host(prev) == ref[log_size]).all()


@pytest.mark.parametrize("log_m", [1, 2, 4, 5, 9, 16])
@pytest.mark.parametrize("fold_step", [1, 2, 3])
def test_fold_line(be, oracle, big_tree, log_m, fold_step):
    if fold_step > log_m:
        pytest.skip("fold_step > log size")
    tree, tw, itw = big_tree
    r = rng(log_m * 10 + fold_step)
    coords = [rand_col(r, log_m) for _ in range(4)]
    alpha = r.integers(0, P, 4, dtype=np.uint32)
    out = be.fold_line(SecureColumn.from_host(coords), alpha, tree, fold_step)
    ref = oracle.fold_line(coords, itw, alpha, fold_step)
    for a, b in zip(out.to_host(), ref):
        assert (a == b).all()


@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 5, 6, 12, 18])
def test_fold_circle_into_line(be, oracle, big_tree, log_n):
    tree, tw, itw = big_tree
    r = rng(300 + log_n)
    src = [rand_col(r, log_n) for _ in range(4)]
    dst = [rand_col(r, log_n - 1) for _ in range(4)]
    alpha = r.integers(0, P, 4, dtype=np.uint32)
    d = SecureColumn.from_host(dst)
    be.fold_circle_into_line(d, SecureColumn.from_host(src), alpha, tree)
    ref = oracle.fold_circle_into_line(dst, src, itw, alpha)
    for a, b in zip(d.to_host(), ref):
        assert (a == b).all()


@pytest.mark.parametrize("log_n", [2, 4, 5, 10, 15])
def test_decompose(be, oracle, log_n):
    r = rng(400 + log_n)
    coords = [rand_col(r, log_n) for _ in range(4)]
    g, lam = be.decompose(SecureColumn.from_host(coords))
    gr, lr = oracle.decompose(coords)
    assert (lam == lr).all()
    for a, b in zip(g.to_host(), gr):
        assert (a == b).all()


def test_throughput_probes_run(be):
    # the register-only ceilings the bench divides by: both launch and finish
    import ctypes as C
    from stwo_b200 import DeviceBuffer, ffi, sync
    out = DeviceBuffer(64)
    ffi.call("stwo_b200_butterfly_probe", C.c_uint32(148), C.c_uint32(4), C.c_void_p(out.ptr), be.stream)
    ffi.call("stwo_b200_blake2s_probe", C.c_uint32(148), C.c_uint32(4), C.c_void_p(out.ptr), be.stream)
    sync(be.stream)
    from stwo_b200.ffi import B200Error
    with pytest.raises(B200Error):
        ffi.call("stwo_b200_butterfly_probe", C.c_uint32(0), C.c_uint32(4), C.c_void_p(out.ptr), be.stream)
