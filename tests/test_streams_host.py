"""Host side of the stream path: the dyadic dissection in librpyb.so and the
CPU restatement of the stream query logic (oracle/streams_ref.py), checked
against the reference's own known answers.  No GPU needed."""
import math

import numpy as np
import pytest

from oracle import streams_ref as R
from roughpy_b200 import _lib

# tests/intervals/test_dyadic_interval.py:217-289 (RealInterval(inf, sup), tol, expected)
KNOWN = [
    ((0.0, 1.0), 1, [(0, 0)]),
    ((0.0, 1.0), 5, [(0, 0)]),
    ((-1.0, 1.0), 1, [(-1, 0), (0, 0)]),
    ((-1.0, 1.5), 1, [(-1, 0), (0, 0), (2, 1)]),
    ((-1.0, 1.25), 1, [(-1, 0), (0, 0)]),
    ((-1.0, 1.25), 2, [(-1, 0), (0, 0), (4, 2)]),
    ((0.0, 1.63451), 1, [(0, 0), (2, 1)]),
    ((0.0, 1.63451), 2, [(0, 0), (2, 1)]),
    ((0.0, 1.63451), 3, [(0, 0), (2, 1), (12, 3)]),
    ((0.0, 1.63451), 7, [(0, 0), (2, 1), (12, 3), (208, 7)]),
]


def lib_dissect(a, b, tol):
    k = np.zeros(256, np.int64)
    p = np.zeros(256, np.int32)
    n = _lib.lib.rpyb_dyadic_dissect(a, b, tol, 1, k.ctypes.data, p.ctypes.data, 256)
    assert n >= 0, _lib.last_error()
    return [(int(k[i]), int(p[i])) for i in range(n)]


@pytest.mark.parametrize("iv,tol,expected", KNOWN)
def test_dissection_known_answers(iv, tol, expected):
    assert lib_dissect(iv[0], iv[1], tol) == expected
    assert R.to_dyadic_intervals(iv[0], iv[1], tol) == expected


def test_dissection_library_matches_restatement_and_tiles_the_interval():
    rng = np.random.default_rng(11)
    for _ in range(3000):
        a, b = np.sort(rng.uniform(-3, 3, size=2))
        tol = int(rng.integers(0, 20))
        pieces = lib_dissect(a, b, tol)
        assert pieces == R.to_dyadic_intervals(a, b, tol)
        # consecutive, and covering [floor(a 2^tol), floor(b 2^tol)) / 2^tol
        lo = math.floor(math.ldexp(a, tol))
        hi = math.floor(math.ldexp(b, tol))
        pos = lo
        for k, p in pieces:
            assert p <= tol
            assert k << (tol - p) == pos
            pos = (k + 1) << (tol - p)
        assert pos == hi or (not pieces and lo == hi)


def test_dissection_walks_match_restatement_over_scales():
    """Both of the library's walks (multipliers below 2^52, and the general one
    between 2^52 and 2^53) against the restatement, over negative and large
    resolutions and interval scales; the batched entry agrees with the single
    one."""
    rng = np.random.default_rng(12)
    cases = []
    for _ in range(3000):
        tol = int(rng.integers(-8, 46))
        top = min(20.0, 58.0 - max(tol, 0))
        scale = 2.0 ** float(rng.uniform(-6.0, top))
        a, b = np.sort(rng.uniform(-scale, scale, size=2))
        cases.append((float(a), float(b), tol))
    for _ in range(300):
        sign = 1.0 if rng.random() < 0.5 else -1.0
        a = sign * float(rng.uniform(4.0, 7.9))
        cases.append((min(a, a + 0.05), max(a, a + 0.05), 50))
    for a, b, tol in cases:
        assert lib_dissect(a, b, tol) == R.to_dyadic_intervals(a, b, tol), (a, b, tol)
    infs = np.array([c[0] for c in cases])
    sups = np.array([c[1] for c in cases])
    tols = np.array([c[2] for c in cases], dtype=np.int32)
    cap = 200 * len(cases)
    k = np.zeros(cap, np.int64)
    p = np.zeros(cap, np.int32)
    off = np.zeros(len(cases) + 1, np.int64)
    assert _lib.lib.rpyb_dyadic_dissect_batch(len(cases), infs.ctypes.data, sups.ctypes.data,
                                              tols.ctypes.data, 1, k.ctypes.data, p.ctypes.data,
                                              cap, off.ctypes.data) == 0
    for i, (a, b, tol) in enumerate(cases[:500]):
        got = [(int(k[j]), int(p[j])) for j in range(off[i], off[i + 1])]
        assert got == lib_dissect(a, b, tol)


def test_batched_dissection_and_errors():
    infs = np.array([0.0, -1.0, 0.5])
    sups = np.array([1.63451, 1.25, 0.5])
    tols = np.array([7, 2, 4], dtype=np.int32)
    k = np.zeros(64, np.int64)
    p = np.zeros(64, np.int32)
    off = np.zeros(4, np.int64)
    assert _lib.lib.rpyb_dyadic_dissect_batch(3, infs.ctypes.data, sups.ctypes.data,
                                              tols.ctypes.data, 1, k.ctypes.data,
                                              p.ctypes.data, 64, off.ctypes.data) == 0
    assert list(off) == [0, 4, 7, 7]
    assert _lib.lib.rpyb_dyadic_dissect(1.0, 0.0, 3, 1, None, None, 0) == _lib.E_INVALID
    assert _lib.lib.rpyb_dyadic_dissect(0.0, 1.0, 3, 0, None, None, 0) == _lib.E_UNSUPPORTED


def arith(golden, w, d):
    g = golden["lie_maps"]
    big = {(2, 2): (2, 4), (2, 3): (2, 4), (2, 4): (2, 4), (3, 2): (3, 3), (3, 3): (3, 3), (4, 2): (4, 3),
           (4, 3): (4, 3)}[(w, d)]
    l2t = g[f"w{big[0]}d{big[1]}_l2t_dense"]
    t2l = g[f"w{big[0]}d{big[1]}_t2l_dense"]
    T = (w ** (d + 1) - 1) // (w - 1)
    L = int(np.count_nonzero(np.abs(l2t[:T]).sum(axis=0)))   # Lie keys of degree <= d
    return R.Arith.from_oracle(w, d, l2t[:T, :L], t2l[:L, :T])


def test_restated_stream_alignment_known_answers(golden):
    # tests/streams/test_lie_increment_path.py:356-382
    a = arith(golden, 3, 2)
    st = R.StreamRef(a, np.array([[0., 1., 2.], [3., 4., 5.]]))
    assert st.resolution == 0
    np.testing.assert_array_equal(st.log_signature(0.0, 0.1)[:3], [0., 1., 2.])
    for i in range(1, 10):
        assert not np.any(st.log_signature(0.1 * i, 0.1 * (i + 1)))
    st4 = R.StreamRef(a, np.array([[0., 1., 2.], [3., 4., 5.]]), resolution=4)
    np.testing.assert_array_equal(st4.log_signature(0.0, 0.1, resolution=4)[:3], [0., 1., 2.])
    for i in range(1, 10):
        assert not np.any(st4.log_signature(0.1 * i, 0.1 * (i + 1), resolution=4))


def test_restated_stream_level_one_sums_and_linear_signature(golden):
    # tests/streams/test_lie_increment_path.py:290-332 and :474-501
    rng = np.random.default_rng(12345)
    arr = rng.integers(0, 5, size=(4, 3)).astype(np.float64)
    a = arith(golden, 3, 2)
    st = R.StreamRef(a, arr)
    sig = st.signature(0.0, 5.0, 2)
    np.testing.assert_array_almost_equal(sig[:4], np.hstack([[1.0], arr.sum(axis=0)]), 12)
    a3 = arith(golden, 3, 3)
    inc = np.array([1., 9., -6.])
    st = R.StreamRef(a3, inc[None, :], indices=np.array([0.0]))
    sig = st.signature(0.0, 1.0)
    l2 = np.einsum("i,j->ij", inc, inc) / 2
    l3 = np.einsum("ij,k->ijk", l2, inc) / 3
    np.testing.assert_array_almost_equal(sig, np.hstack([[1.0], inc, l2.ravel(), l3.ravel()]))


def test_restated_sig_derivative_known_answers(golden):
    # tests/streams/test_lie_increment_path.py:233-263: one tick [0.2, 0.4, 0.6],
    # perturbation e_2, interval [0, 1)
    a = arith(golden, 3, 2)
    got = a.sig_derivative([(np.array([0.2, 0.4, 0.6, 0.0, 0.0, 0.0]),
                             np.array([0.0, 1.0, 0.0, 0.0, 0.0, 0.0]))])
    want = np.array([0.0, 0.0, 1.0, 0.0, 0.0, 0.1, 0.0, 0.1, 0.4, 0.3, 0.0, 0.3, 0.0])
    assert np.max(np.abs(got - want)) <= 1e-15


@pytest.mark.parametrize("count", [1, 2, 5])
def test_restated_piecewise_full_data_is_cbh_of_the_pieces(golden, count):
    # tests/streams/test_piecewise_lie_path.py:41-51: log_signature at
    # resolution 5 over unit pieces [i, i+1) equals the CBH of all pieces
    a = arith(golden, 4, 3)
    rng = np.random.default_rng(count)
    lies = []
    for _ in range(count):
        v = np.zeros(a.L)
        v[:4] = rng.normal(0.0, 1.0, 4)
        lies.append(v)
    st = R.PiecewiseRef(a, [(float(i), float(i + 1), v) for i, v in enumerate(lies)])
    np.testing.assert_array_almost_equal(st.log_signature(resolution=5), a.cbh(lies), decimal=12)


def test_tick_restatement_known_answer(golden):
    """Two increments at one time step, combined by CBH in input order
    (tests/streams/test_tick_stream.py:107-115 expects Lie([1, 1, 0.5]) for
    "first" then "second"); the reverse order flips the bracket."""
    a = arith(golden, 2, 2)
    e1, e2 = [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]
    t = R.TickRef(a, [(1.0, e1), (1.0, e2)], resolution=0, support=(0.0, 2.0))
    np.testing.assert_allclose(t.log_signature(0.0, 2.0, 2), [1.0, 1.0, 0.5], atol=1e-15)
    t = R.TickRef(a, [(1.0, e2), (1.0, e1)], resolution=0, support=(0.0, 2.0))
    np.testing.assert_allclose(t.log_signature(0.0, 2.0, 2), [1.0, 1.0, -0.5], atol=1e-15)


@pytest.mark.parametrize("w,d", [(2, 3), (3, 3)])
def test_tick_restatement_matches_the_cached_stream_on_distinct_times(golden, w, d):
    """With one event per leaf, in time order, the tick stream's compressed
    recursion and the caching layer's cached leaves give the same
    log-signatures on every query (both are the CBH of the events inside)."""
    a = arith(golden, w, d)
    rng = np.random.default_rng(w + 10 * d)
    res = 4
    # no event in the leaf at 0 next to negative ones (the reference's
    # construction does not end for that case)
    cand = np.concatenate([np.arange(-20, 0), np.arange(1, 40)])
    leaves = np.sort(rng.choice(cand, size=15, replace=False))
    times = leaves / 2.0 ** res + rng.uniform(0, 1, 15) / 2.0 ** (res + 1)
    rows = rng.normal(0, 0.3, (15, a.L))
    support = (float(times.min()), float(times.max()) + 2.0 ** -res)
    tick = R.TickRef(a, [(t, r) for t, r in zip(times, rows)], resolution=res, support=support)
    ref = R.StreamRef(a, rows, indices=times, resolution=res)
    ref.support = support
    for _ in range(30):
        lo, hi = np.sort(rng.uniform(support[0] - 0.2, support[1] + 0.2, 2))
        for q_res in (None, res - 2, res + 2):
            np.testing.assert_allclose(tick.log_signature(lo, hi, q_res),
                                       ref.log_signature(lo, hi, q_res), atol=1e-12)


def test_tick_restatement_rejects_events_on_both_sides_of_zero_leaf(golden):
    """The reference's search for the smallest dyadic interval holding events
    before 0 and in the leaf at 0 never ends (k stays -1); the restatement
    raises instead."""
    a = arith(golden, 2, 2)
    with pytest.raises(ValueError):
        R.TickRef(a, [(-0.5, [1.0, 0.0, 0.0]), (0.25, [0.0, 1.0, 0.0])], resolution=0)


def test_tick_stream_event_layout_for_the_tree():
    """TickStream.from_lie_events (host side, nothing on the device until the
    first query): events are ordered stably by their dyadic interval at the
    stream resolution, keep their input order inside an interval (no
    de-duplication by time) and sit at the interval's start; the defaults
    are resolution 0 and support [0, 1); bad inputs are rejected."""
    from roughpy_b200.streams import TickStream
    times = [0.30, 0.10, 0.27, 0.26, -0.05, 0.10]
    rows = np.arange(12.0).reshape(6, 2)
    st = TickStream.from_lie_events(times, rows, 2, 2, resolution=2, support=(-1.0, 1.0))
    # intervals at resolution 2: 1, 0, 1, 1, -1, 0
    np.testing.assert_array_equal(st.times, [-0.25, 0.0, 0.0, 0.25, 0.25, 0.25])
    np.testing.assert_array_equal(st.lies[:, :2], rows[[4, 1, 5, 0, 2, 3]])
    assert (st.support.inf, st.support.sup) == (-1.0, 1.0)
    st = TickStream.from_lie_events([0.5], [[1.0, 2.0]], 2, 2)
    assert st.resolution == 0 and (st.support.inf, st.support.sup) == (0.0, 1.0)
    with pytest.raises(ValueError):
        TickStream.from_lie_events([0.1, 0.2], [[1.0, 2.0]], 2, 2)
    with pytest.raises(ValueError):
        TickStream.from_lie_events([], np.zeros((0, 2)), 2, 2)
    with pytest.raises(NotImplementedError):
        TickStream.from_data({1.0: [("a", "increment", 1.0)]}, width=2, depth=2)
    with pytest.raises(TypeError):
        TickStream.from_increments(rows, width=2, depth=2)


def test_partition_and_restrict_host_side():
    """Partition keeps the points strictly inside, sorted, duplicates
    included (intervals/src/partition.cpp:45-56, :93-110); restrict replaces
    the support without touching the events, and the restricted copy
    rebuilds its device tree (nothing is built here)."""
    from roughpy_b200.streams import LieIncrementStream, Partition, RealInterval
    p = Partition(RealInterval(0.0, 1.0), [0.75, 0.25, 1.0, 0.0, 1.5, 0.25])
    assert p.intermediates() == [0.25, 0.25, 0.75]
    assert len(p) == 4
    assert [(p[i].inf, p[i].sup) for i in range(4)] == [(0.0, 0.25), (0.25, 0.25), (0.25, 0.75),
                                                       (0.75, 1.0)]
    assert p.mesh() == 0.5
    assert Partition((0.0, 1.0))[0].sup == 1.0
    assert Partition((0.0, 1.0), [0.5]).refine_midpoints().intermediates() == [0.25, 0.5, 0.75]
    st = LieIncrementStream.from_increments(np.ones((4, 2)), width=2, depth=2)
    r = st.restrict(RealInterval(1.0, 2.5))
    assert (r.support.inf, r.support.sup) == (1.0, 2.5)
    assert (st.support.inf, st.support.sup) == (0.0, 4.0)
    assert r._tree is None and r.lies is st.lies
    assert r.restrict((0.0, 9.0))._base_support is st.support


def test_partition_reference_cases():
    """tests/intervals/test_partitions.py:9-23: intermediates outside the
    interval (or at its ends) are dropped; a pickle round trip compares
    equal."""
    import pickle
    from roughpy_b200.streams import Partition, RealInterval
    assert Partition(RealInterval(0.0, 1.0), intermediates=np.arange(10)).intermediates() == []
    p = Partition(RealInterval(0.5, 1.6), [0.9, 1.3])
    assert pickle.loads(pickle.dumps(p)) == p
    assert p != Partition(RealInterval(0.5, 1.6), [0.9])


def test_query_argument_rules():
    """signature_arguments.cpp:30-50 and :95-170: a float resolution is an
    accuracy (param_to_resolution), after an interval the second argument is
    the resolution, a float alone is rejected, and sup must be a number."""
    from roughpy_b200.streams import (LieIncrementStream, RealInterval, _resolution_arg,
                                      param_to_resolution)
    assert _resolution_arg(None) is None
    assert _resolution_arg(3) == 3 and _resolution_arg(np.int32(4)) == 4
    assert _resolution_arg(0.5) == param_to_resolution(0.5) == 1
    assert _resolution_arg(0.25) == 2 and _resolution_arg(np.float64(1e-3)) == 10
    assert _resolution_arg(100.0) == -5   # coarse accuracies stop at resolution -5
    with pytest.raises(TypeError):
        _resolution_arg("4")
    with pytest.raises(TypeError):
        _resolution_arg(True)
    st = LieIncrementStream.from_increments(np.ones((4, 2)), width=2, depth=2)
    assert st._interval_args(RealInterval(0.0, 1.0), 3) == (0.0, 1.0, 3)
    assert st._interval_args(RealInterval(0.0, 1.0), 0.25) == (0.0, 1.0, 2)
    assert st._interval_args(0.0, 0.8, 0.5) == (0.0, 0.8, 1)
    assert st._interval_args(5, None) == (0.0, 4.0, 5)
    assert st._interval_args(None, None, 0.125) == (0.0, 4.0, 3)
    with pytest.raises(TypeError):
        st._interval_args(0.5, None)
    with pytest.raises(TypeError):
        st._interval_args(0.0, "1")
    with pytest.raises(ValueError):
        st._interval_args(1.0, 0.0)


def test_restated_stream_accuracy_arguments(golden):
    """tests/streams/test_lie_increment_path.py:132-143: one tick at 0.7;
    accuracy 0.5 (resolution 1) sees nothing in [0, 0.8), accuracy 0.25
    (resolution 2) sees the tick."""
    from roughpy_b200.streams import param_to_resolution
    a = arith(golden, 2, 2)
    st = R.StreamRef(a, np.array([[1.0, 2.5]]), indices=np.array([0.7]))
    unit = np.zeros(a.T)
    unit[0] = 1.0
    np.testing.assert_array_equal(st.signature(0.0, 0.8, param_to_resolution(0.5)), unit)
    np.testing.assert_allclose(st.signature(0.0, 0.8, param_to_resolution(0.25)),
                               [1.0, 1.0, 2.5, 0.5, 1.25, 1.25, 3.125], atol=1e-15)


def _straight_line_signature(w, d, length):
    """The signature of a straight line with increment length * (1, ..., w):
    level k holds prod(word) * length^k / k! (tests/streams/
    test_lie_increment_path.py:171-195, solution_signature)."""
    import itertools
    out = [1.0]
    for k in range(1, d + 1):
        for word in itertools.product(range(1, w + 1), repeat=k):
            out.append(float(np.prod(word)) * length ** k / math.factorial(k))
    return np.array(out)


@pytest.mark.parametrize("w,d", [(2, 2), (2, 4), (3, 3), (4, 3)])
@pytest.mark.parametrize("n", [2, 5, 10, 25, 100])
def test_restated_stream_known_straight_line_signature(golden, w, d, n):
    """tests/streams/test_lie_increment_path.py:160-205: n equal increments
    2/n * (1, ..., w) at t = 2/n, 4/n, ..., 2; the signature over [0, 3.125)
    is that of the straight line over [0, 2]."""
    a = arith(golden, w, d)
    t_values = np.arange(0.0, 2.0, 2.0 / n) + 2.0 / n
    data = np.tensordot(np.ones(n), np.arange(1.0, w + 1) * (2.0 / n), axes=0)
    st = R.StreamRef(a, data, indices=t_values)
    np.testing.assert_allclose(st.signature(0.0, 3.125), _straight_line_signature(w, d, 2.0),
                               rtol=1e-12, atol=1e-12)


def test_restated_stream_signature_multiplication(golden):
    """tests/streams/test_lie_increment_path.py:386-399 (float64 here):
    the signatures over [0, pi/4) and [pi/4, 2) multiply to the one over
    [0, 2)."""
    import oracle
    a = arith(golden, 3, 2)
    data = np.array([[0., 1., 2.], [3., 4., 5.], [6., 7., 8.]])
    st = R.StreamRef(a, data, indices=np.array([0., np.pi / 4, 1.0]))
    left = st.signature(0.0, np.pi / 4)
    right = st.signature(np.pi / 4, 2.0)
    full = st.signature(0.0, 2.0)
    np.testing.assert_allclose(oracle.ft_mul(3, 2, left, right), full, rtol=1e-12, atol=1e-12)


def test_restated_stream_of_lie_elements(golden):
    """tests/streams/test_lie_increment_path.py:401-413: a sequence of Lie
    elements at t = 0, 1, 2; the log-signature over [0, 1) is the first."""
    a = arith(golden, 3, 3)
    seq = np.array([[1., 2., 3.], [4., 5., 6.], [7., 8., 9.]])
    st = R.StreamRef(a, seq)
    lie = st.log_signature(0.0, 1.0)
    np.testing.assert_array_equal(lie[:3], seq[0])
    assert not np.any(lie[3:])


def test_simplify_argument_rules_follow_the_binding():
    """roughpy/src/streams/stream.cpp:410-468: resolution and depth are C ints
    (a float is a TypeError), a context takes precedence over depth and must
    have the stream's width.  A depth above the stream's is rejected (the
    device tree holds the stream's depth).  All checks run on the host before
    any device work."""
    import types
    from roughpy_b200.streams import LieIncrementStream, Partition, RealInterval
    st = LieIncrementStream.from_increments(np.zeros((4, 3)), width=3, depth=3)
    part = Partition(RealInterval(0.0, 1.0), [0.5])
    with pytest.raises(TypeError):
        st.simplify(part, resolution=2.0)
    with pytest.raises(TypeError):
        st.simplify(part, depth=2.5)
    with pytest.raises(ValueError, match="width"):
        st.simplify(part, ctx=types.SimpleNamespace(width=2, depth=2))
    with pytest.raises(ValueError, match="exceeds"):
        st.simplify(part, depth=4)
    # the context wins over depth: a valid depth does not rescue a bad context
    with pytest.raises(ValueError, match="exceeds"):
        st.simplify(part, ctx=types.SimpleNamespace(width=3, depth=5), depth=2)
