"""GPU stream queries (roughpy_b200.streams) against the reference's stream
semantics: golden fixtures computed with the reference's own arithmetic through
the restated DyadicCachingLayer, the restatement itself on random streams, and
the reference test suite's known answers.

Tolerances: signatures (float64 tree) <= 1e-12 per-level relative; log
signatures are compared with an absolute floor of 1e-12 x the level scale,
because exact-zero levels (e.g. a single event) make a relative error
meaningless.  The float32-compensated tree is held to 1e-6."""
import numpy as np
import pytest

from oracle import streams_ref as R
from roughpy_b200.streams import LieIncrementStream, RealInterval
from tests._util import level_rel_err

pytestmark = pytest.mark.gpu


def lie_close(got, want, tol):
    scale = max(1.0, float(np.max(np.abs(want))))
    assert float(np.max(np.abs(np.asarray(got) - want))) <= tol * scale


@pytest.mark.parametrize("tag", ["a", "b", "c", "d"])
def test_queries_match_reference_golden(golden, tag):
    g = golden["streams"]
    w, d, res = (int(v) for v in g[f"{tag}_meta"])
    idx = g[f"{tag}_idx"]
    st = LieIncrementStream.from_increments(g[f"{tag}_inc"], indices=None if idx.size == 0 else idx,
                                            width=w, depth=d,
                                            resolution=None if res < 0 else res)
    assert st.resolution == int(g[f"{tag}_resolution"][0])
    q = g[f"{tag}_queries"]
    lie = st.log_signature_batch(q[:, 0], q[:, 1]).cpu().numpy()
    sig = st.signature_batch(q[:, 0], q[:, 1]).cpu().numpy()
    lie_close(lie, g[f"{tag}_logsig"], 1e-12)
    assert level_rel_err(sig, g[f"{tag}_sig"], w, d) <= 1e-12
    # single-query API agrees with the batch
    for i in (0, 4, 7):
        lie_close(st.log_signature(q[i, 0], q[i, 1]), g[f"{tag}_logsig"][i], 1e-12)


def _arith(golden, w, d):
    from tests.test_streams_host import arith
    return arith(golden, w, d)


@pytest.mark.parametrize("w,d,n,res", [(2, 4, 200, 7), (3, 3, 150, None), (4, 2, 300, 4),
                                       (3, 3, 90, 9)])
def test_random_streams_against_restatement(golden, w, d, n, res):
    rng = np.random.default_rng(w * 100 + n)
    inc = rng.normal(0, 0.2, size=(n, w))
    idx = np.sort(rng.uniform(-0.5, 1.5, size=n))
    ref = R.StreamRef(_arith(golden, w, d), inc, idx, res)
    st = LieIncrementStream.from_increments(inc, indices=idx, width=w, depth=d, resolution=res)
    assert st.resolution == ref.resolution
    qs = np.sort(rng.uniform(-0.7, 1.7, size=(25, 2)), axis=1)
    got = st.signature_batch(qs[:, 0], qs[:, 1]).cpu().numpy()
    want = np.stack([ref.signature(a, b) for a, b in qs])
    assert level_rel_err(got, want, w, d) <= 1e-12
    # explicit coarse and fine query resolutions
    for qres in (2, ref.resolution + 3):
        got = st.log_signature_batch(qs[:8, 0], qs[:8, 1], resolution=qres).cpu().numpy()
        want = np.stack([ref.log_signature(a, b, qres) for a, b in qs[:8]])
        lie_close(got, want, 1e-11)


def test_reference_known_answers():
    # tests/streams/test_lie_increment_path.py:96-130
    s = LieIncrementStream.from_increments(np.array([[3, 7, 0], [0, 0, 1]]), depth=2,
                                           coeffs="DPReal")
    np.testing.assert_array_equal(s.signature(depth=1), [1, 3, 7, 1])
    s = LieIncrementStream.from_increments(np.array([[3, 7, 0, 4], [0, 0, 1, 5]]), width=2,
                                           depth=2)
    np.testing.assert_array_equal(s.signature(depth=1), [1, 3, 7])
    # :356-382 alignment with default and explicit resolution
    s = LieIncrementStream.from_increments(np.array([[0., 1., 2.], [3., 4., 5.]]), depth=2)
    np.testing.assert_array_equal(s.log_signature(RealInterval(0.0, 0.1))[:3], [0., 1., 2.])
    for i in range(1, 10):
        assert not np.any(s.log_signature(RealInterval(0.1 * i, 0.1 * (i + 1))))
    s = LieIncrementStream.from_increments(np.array([[0., 1., 2.], [3., 4., 5.]]), depth=2,
                                           resolution=4)
    np.testing.assert_array_equal(s.log_signature(RealInterval(0.0, 0.1), resolution=4)[:3],
                                  [0., 1., 2.])
    # :290-332 level one is the sum of the increments
    rng = np.random.default_rng(12345)
    arr = rng.integers(0, 5, size=(4, 3))
    s = LieIncrementStream.from_increments(arr, width=3, depth=2)
    np.testing.assert_array_almost_equal(s.signature(RealInterval(0.0, 5.0), resolution=2)[:4],
                                         np.hstack([[1.0], arr.sum(axis=0)]), 13)
    s = LieIncrementStream.from_increments(arr.T, width=4, depth=2)
    np.testing.assert_array_almost_equal(s.signature(RealInterval(0.0, 5.0))[:5],
                                         np.hstack([[1.0], arr.sum(axis=1)]), 13)
    # :474-501 one increment: the signature is exp(increment)
    inc = np.array([1., 9., -6.])
    s = LieIncrementStream.from_increments(inc[None, :], indices=np.array([0.0]), width=3,
                                           depth=3)
    l2 = np.einsum("i,j->ij", inc, inc) / 2
    l3 = np.einsum("ij,k->ijk", l2, inc) / 3
    np.testing.assert_array_almost_equal(s.signature(RealInterval(0., 1.)),
                                         np.hstack([[1.0], inc, l2.ravel(), l3.ravel()]))


def test_tree_like_paths_have_the_pruned_signature():
    # tests/streams/test_lie_increment_path.py:427-471
    def sig(path, depth=2):
        inc = np.diff(np.asarray(path, dtype=np.float64), axis=0)
        if inc.shape[0] == 0:
            inc = np.zeros((1, 2))
        return LieIncrementStream.from_increments(inc, width=2, depth=depth).signature()
    tree_like = [[0.0, 0], [1, 3], [0, 0], [1, 5], [2, 5], [1, 5], [0, 6], [1, 5], [0, 0]]
    np.testing.assert_array_almost_equal(sig(tree_like), sig([[0., 0.], [0., 0.]]))
    tree_like = [[0.0, 0], [1, 1], [3, 1], [2, 1], [1, 1], [2, 0]]
    np.testing.assert_array_almost_equal(sig(tree_like), sig([[0., 0.], [1., 1.], [2., 0]]))


def test_general_lie_increments_use_the_exponential_path(golden):
    # rows with bracket coordinates: leaves are products of exp(l2t(lie))
    rng = np.random.default_rng(4)
    lies = rng.normal(0, 0.3, size=(12, 3))          # (2,2) Lie dimension 3
    idx = np.arange(12) / 8.0
    ref = R.StreamRef(_arith(golden, 2, 2), lies, idx, 2)
    st = LieIncrementStream.from_increments(lies, indices=idx, width=2, depth=2, resolution=2)
    qs = np.array([[0.0, 1.5], [0.1, 0.9], [0.25, 0.5]])
    got = st.signature_batch(qs[:, 0], qs[:, 1]).cpu().numpy()
    want = np.stack([ref.signature(a, b) for a, b in qs])
    assert level_rel_err(got, want, 2, 2) <= 1e-12


def test_dyadic_queries_float32_tree_within_1e6():
    """The dyadic-query workload shape at reduced size: 2^12 events at t_i = i 2^-12,
    width 6, depth 5, resolution 12, queries rounded to the resolution."""
    n = 1 << 12
    rng = np.random.default_rng(3)
    inc = rng.normal(0, np.sqrt(1.0 / n), size=(n, 6))
    idx = np.arange(n) / n
    q = np.sort(np.floor(rng.uniform(0, 1, size=(300, 2)) * n) / n, axis=1)
    s64 = LieIncrementStream.from_increments(inc, indices=idx, width=6, depth=5, resolution=12)
    s32 = LieIncrementStream.from_increments(inc.astype(np.float32), indices=idx, width=6,
                                             depth=5, resolution=12)
    assert s32.mode == "f32c"
    sig64 = s64.signature_batch(q[:, 0], q[:, 1]).cpu().numpy()
    sig32 = s32.signature_batch(q[:, 0], q[:, 1]).cpu().numpy()
    # full-interval signature equals the plain Chen product of all increments
    import oracle
    full = s64.signature(0.0, 1.0)
    assert level_rel_err(full, oracle.signature(6, 5, inc), 6, 5) <= 1e-11
    # f32 tree against the f64 tree, same (float32-rounded) increments
    s64b = LieIncrementStream.from_increments(inc.astype(np.float32).astype(np.float64),
                                              indices=idx, width=6, depth=5, resolution=12)
    ref = s64b.signature_batch(q[:, 0], q[:, 1]).cpu().numpy()
    assert level_rel_err(sig32, ref, 6, 5) <= 1e-6
    assert sig64.shape == sig32.shape


def _build_raw(mode, w, d, res, s0, s1, times, rows):
    """rpyb_dyadic_build called directly through the C ABI."""
    import ctypes
    import torch
    from roughpy_b200 import _lib
    h = ctypes.c_void_p()
    _lib.check(_lib.lib.rpyb_dyadic_build(mode, w, d, res, s0, s1, len(times),
                                          times.ctypes.data, rows.data_ptr(), rows.shape[1],
                                          ctypes.byref(h), torch.cuda.current_stream().cuda_stream))
    return h


def test_c_abi_tree_nodes_are_chen_products_of_their_leaves():
    """Every node of rpyb_dyadic_build's tree equals the signature of the events
    inside its dyadic interval (computed by the batched signature kernel), and
    the top node over a support inside [0, 1) is the whole stream's signature."""
    import ctypes
    import torch
    from roughpy_b200 import _lib
    from roughpy_b200 import signatures as S
    rng = np.random.default_rng(11)
    w, d, res, n = 3, 4, 4, 37
    times = np.sort(rng.uniform(0, 1, n))
    inc = torch.from_numpy(rng.normal(0, 0.3, (n, w))).cuda()
    h = _build_raw(_lib.F64, w, d, res, 0.0, 1.0, times, inc)
    try:
        rows, top, nodes = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_void_p()
        _lib.check(_lib.lib.rpyb_dyadic_tree_info(h, ctypes.byref(rows), ctypes.byref(top),
                                                  ctypes.byref(nodes)))
        T = S.tensor_size(w, d)
        assert top.value == res
        for level in range(res + 1):
            for blk in range(2 ** (res - level)):
                r = int(_lib.lib.rpyb_dyadic_node_row(h, level, blk))
                assert r >= 0
                lo, hi = blk * 2.0 ** (level - res), (blk + 1) * 2.0 ** (level - res)
                sel = (times >= lo) & (times < hi)
                want = S.signature(inc[torch.from_numpy(sel).cuda()], None, d, "f64")[0]
                torch.cuda.synchronize()
                got = _node(nodes.value, r, T)
                assert level_rel_err(got, want.cpu().numpy(), w, d) <= 1e-13
        assert int(_lib.lib.rpyb_dyadic_node_row(h, res + 1, 0)) == -1
        assert int(_lib.lib.rpyb_dyadic_node_row(h, 0, 2 ** res)) == -1
    finally:
        _lib.lib.rpyb_dyadic_free(h)


def _node(ptr, row, T):
    """Copy one float64 tree row from device memory to the host."""
    import ctypes
    from roughpy_b200 import _lib
    host = np.empty(T, dtype=np.float64)
    # cudaMemcpy resolved through librpyb's own CUDA runtime dependency
    copy = _lib.lib.cudaMemcpy
    copy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    copy.restype = ctypes.c_int
    assert copy(host.ctypes.data, ptr + row * T * 8, T * 8, 2) == 0   # device to host
    return host


def test_c_abi_query_outputs_agree_and_reject_bad_intervals():
    """rpyb_dyadic_query: log-signature alone, signature alone and both at once
    agree; the signature is exp(l2t(logsig)); an interval with inf > sup is
    rejected with RPYB_E_INVALID."""
    import torch
    from roughpy_b200 import _lib
    from roughpy_b200 import compute as rpc
    rng = np.random.default_rng(12)
    w, d, res, n = 2, 5, 6, 90
    times = np.sort(rng.uniform(-0.5, 1.5, n))
    inc = torch.from_numpy(rng.normal(0, 0.2, (n, w))).cuda()
    h = _build_raw(_lib.F64, w, d, res, -0.5, 1.5, times, inc)
    try:
        q = np.sort(rng.uniform(-0.7, 1.7, (25, 2)), axis=1)
        a, b = np.ascontiguousarray(q[:, 0]), np.ascontiguousarray(q[:, 1])
        L, T = rpc.LieBasis(w, d).size(), rpc.TensorBasis(w, d).size()
        s = torch.cuda.current_stream().cuda_stream
        l1 = torch.empty((25, L), dtype=torch.float64, device="cuda")
        s1 = torch.empty((25, T + 3), dtype=torch.float64, device="cuda")
        l2 = torch.empty_like(l1)
        s2 = torch.empty((25, T), dtype=torch.float64, device="cuda")
        A = _lib.QUERY_RESOLUTION_AUTO
        _lib.check(_lib.lib.rpyb_dyadic_query(h, 25, a.ctypes.data, b.ctypes.data, A,
                                              l1.data_ptr(), L, None, 0, s))
        _lib.check(_lib.lib.rpyb_dyadic_query(h, 25, a.ctypes.data, b.ctypes.data, A,
                                              None, 0, s1.data_ptr(), T + 3, s))
        _lib.check(_lib.lib.rpyb_dyadic_query(h, 25, a.ctypes.data, b.ctypes.data, A,
                                              l2.data_ptr(), L, s2.data_ptr(), T, s))
        assert torch.equal(l1, l2)
        assert torch.equal(s1[:, :T], s2)
        emb = torch.zeros((25, T), dtype=torch.float64, device="cuda")
        rpc._internals.dense_lie_to_tensor(emb, l1, rpc.LieBasis(w, d).get_l2t_matrix(),
                                           rpc.LieBasis(w, d), rpc.TensorBasis(w, d))
        ex = torch.zeros_like(emb)
        rpc._internals.dense_ft_exp(ex, emb, rpc.TensorBasis(w, d))
        assert float((ex - s2).abs().max()) <= 1e-13 * float(s2.abs().max())
        bad_a, bad_b = np.array([0.5]), np.array([0.25])
        rc = _lib.lib.rpyb_dyadic_query(h, 1, bad_a.ctypes.data, bad_b.ctypes.data, A,
                                        l1.data_ptr(), L, None, 0, s)
        assert rc == _lib.E_INVALID
        rc = _lib.lib.rpyb_dyadic_query(h, 1, a.ctypes.data, b.ctypes.data, A, None, 0, None, 0, s)
        assert rc == _lib.E_INVALID
    finally:
        _lib.lib.rpyb_dyadic_free(h)


def test_c_abi_build_rejects_unsorted_times_and_bad_rows():
    import ctypes
    import torch
    from roughpy_b200 import _lib
    h = ctypes.c_void_p()
    t = np.array([0.5, 0.25])
    rows = torch.zeros((2, 3), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert _lib.lib.rpyb_dyadic_build(_lib.F64, 3, 3, 2, 0.0, 1.0, 2, t.ctypes.data,
                                      rows.data_ptr(), 3, ctypes.byref(h), s) == _lib.E_INVALID
    t = np.array([0.25, 0.5])
    assert _lib.lib.rpyb_dyadic_build(_lib.F64, 3, 3, 2, 0.0, 1.0, 2, t.ctypes.data,
                                      rows.data_ptr(), 4, ctypes.byref(h), s) == _lib.E_INVALID
    assert not h.value


@pytest.mark.parametrize("w,d", [(2, 12), (3, 8), (4, 6), (5, 4), (8, 4), (6, 5)])
def test_c_abi_query_signatures_are_chen_products_of_events(w, d):
    """Queries on the tree's grid (one or two top-level units per thread of the
    fused chain-product kernel, widths 2..8): the signature of [a, b) equals
    the signature of the events inside it, computed by the batched signature
    kernel, and the log-signature equals t2l(log) of that signature; an empty
    interval gives the unit and a zero log-signature."""
    import torch
    from roughpy_b200 import _lib
    from roughpy_b200 import compute as rpc
    from roughpy_b200 import signatures as S
    rng = np.random.default_rng(w * 31 + d)
    res, n = 6, 80
    times = np.sort(rng.uniform(0, 1, n))
    inc = torch.from_numpy(rng.normal(0, 0.05, (n, w))).cuda()
    h = _build_raw(_lib.F64, w, d, res, 0.0, 1.0, times, inc)
    try:
        T = S.tensor_size(w, d)
        lb, tb = rpc.LieBasis(w, d), rpc.TensorBasis(w, d)
        L = lb.size()
        grid = np.sort(rng.integers(0, 2 ** res + 1, (12, 2)), axis=1) / 2.0 ** res
        grid[0] = [0.25, 0.25]
        a, b = np.ascontiguousarray(grid[:, 0]), np.ascontiguousarray(grid[:, 1])
        sig = torch.empty((12, T), dtype=torch.float64, device="cuda")
        lie = torch.empty((12, L), dtype=torch.float64, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        _lib.check(_lib.lib.rpyb_dyadic_query(h, 12, a.ctypes.data, b.ctypes.data, res,
                                              lie.data_ptr(), L, sig.data_ptr(), T, s))
        got = sig.cpu().numpy()
        unit = np.zeros(T)
        unit[0] = 1.0
        assert np.array_equal(got[0], unit)
        assert not lie[0].any()
        wants = []
        for i in range(12):
            sel = (times >= a[i]) & (times < b[i])
            if not sel.any():
                wants.append(torch.from_numpy(unit).cuda())
                assert np.abs(got[i] - unit).max() <= 1e-13
                continue
            want = S.signature(inc[torch.from_numpy(sel).cuda()], None, d, "f64")[0]
            wants.append(want)
            wn = want.cpu().numpy()
            if d <= 8:
                assert level_rel_err(got[i], wn, w, d) <= 1e-11, i
            else:
                # At depth 12 the top levels (~1e-13) come out of the log's
                # Horner terms (~r^k, r the l1 norm of the non-scalar part) by
                # cancellation, so the float64 log -> exp round trip is accurate
                # to ~eps r^k there, not to the level's own size: bound each
                # level's absolute error by 1e-13 r^k.  A wrong word would be
                # off by the level's size, far above the bound.
                r = float(np.abs(wn[1:]).sum())
                db = [0]
                for _ in range(d + 1):
                    db.append(1 + w * db[-1])
                for k in range(d + 1):
                    err = np.abs(got[i, db[k]:db[k + 1]] - wn[db[k]:db[k + 1]]).max()
                    assert err <= 1e-13 * max(r, 1e-3) ** k, (i, k, err)
        # log-signatures: t2l(log(signature of the events))
        W = torch.stack(wants)
        lg = torch.zeros_like(W)
        rpc._internals.dense_ft_log(lg, W, tb)
        ref = torch.zeros((12, L), dtype=torch.float64, device="cuda")
        rpc._internals.dense_tensor_to_lie(ref, lg, lb.get_t2l_matrix(), lb, tb)
        scale = max(float(ref.abs().max()), 1e-300)
        assert float((lie - ref).abs().max()) <= 1e-11 * scale
    finally:
        _lib.lib.rpyb_dyadic_free(h)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_saved_stream_tree_loads_and_answers_identically(tmp_path, dtype):
    """LieIncrementStream.save / load (rpyb_dyadic_save / rpyb_dyadic_load):
    the loaded tree gives bit-identical query results, and damaged blocks are
    rejected on the host before anything reaches the device."""
    import ctypes
    import torch
    from roughpy_b200 import _lib
    rng = np.random.default_rng(77)
    n = 700
    inc = rng.normal(0, 0.1, size=(n, 4)).astype(dtype)
    idx = np.sort(rng.uniform(-0.3, 1.2, size=n))
    st = LieIncrementStream.from_increments(inc, indices=idx, width=4, depth=4, resolution=9)
    q = np.sort(rng.uniform(-0.5, 1.5, size=(64, 2)), axis=1)
    want_lie = st.log_signature_batch(q[:, 0], q[:, 1]).cpu()
    want_sig = st.signature_batch(q[:, 0], q[:, 1]).cpu()
    path = tmp_path / "stream.npz"
    st.save(path)
    back = LieIncrementStream.load(path)
    assert (back.width, back.depth, back.resolution, back.mode) == (4, 4, 9, st.mode)
    assert back.support.inf == st.support.inf and back.support.sup == st.support.sup
    assert back._tree.rows == st._tree.rows and back._tree.top_level == st._tree.top_level
    assert torch.equal(back.log_signature_batch(q[:, 0], q[:, 1]).cpu(), want_lie)
    assert torch.equal(back.signature_batch(q[:, 0], q[:, 1]).cpu(), want_sig)
    # damaged blocks
    blob = np.ascontiguousarray(np.load(path)["tree"])
    h = ctypes.c_void_p()
    s = torch.cuda.current_stream().cuda_stream
    bad = blob.copy()
    bad[0] ^= 0xFF
    assert _lib.lib.rpyb_dyadic_load(bad.ctypes.data, bad.size, ctypes.byref(h), s) == \
        _lib.E_INVALID
    short = blob[:-8].copy()
    assert _lib.lib.rpyb_dyadic_load(short.ctypes.data, short.size, ctypes.byref(h), s) == \
        _lib.E_INVALID
    assert not h.value
    from roughpy_b200.streams import TickStream
    with pytest.raises(TypeError):
        TickStream.load(path)


@pytest.mark.parametrize("w,d", [(2, 4), (3, 3), (4, 3)])
def test_batched_cbh_against_the_restated_context(golden, w, d):
    """rpyb_cbh (roughpy_b200.streams.cbh_batch) against the restated
    Context::cbh (algebra/src/context.cpp:187-208) on lists of 0, 1, 2 and 7
    Lie elements, including a zero element; a single element comes back
    unchanged."""
    from roughpy_b200.streams import cbh, cbh_batch
    a = _arith(golden, w, d)
    rng = np.random.default_rng(w * 10 + d)
    sizes = [2, 0, 1, 7, 3]
    lists = [[rng.normal(0, 0.3, size=a.L) for _ in range(k)] for k in sizes]
    lists[3][2] = np.zeros(a.L)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    flat = np.array([x for lst in lists for x in lst])
    got = cbh_batch(flat, off, w, d).cpu().numpy()
    for q, lst in enumerate(lists):
        want = a.cbh(lst) if lst else np.zeros(a.L)
        lie_close(got[q], want, 1e-12)
    assert np.array_equal(got[2], lists[2][0])
    lie_close(cbh(lists[0], w, d), a.cbh(lists[0]), 1e-12)


@pytest.mark.parametrize("dtype,n,res,lo", [(np.float64, 5000, 12, 0.0), (np.float32, 6000, 12, -0.4),
                                            (np.float64, 3000, 13, -1.0)])
def test_range_table_queries_equal_the_piece_products(dtype, n, res, lo):
    """rpyb_dyadic_range_table: queries answered from the table (at most four
    rows) equal the piece-by-piece products of the same tree: float64 trees
    to 1e-12 (the product is only reassociated), float32 trees to 1e-6.
    Queries include block-aligned ends, ranges inside one block, empty and
    out-of-support ranges, supports on both sides of 0, and resolutions finer
    than the stream's (those keep the piece path)."""
    rng = np.random.default_rng(n + res)
    inc = rng.normal(0, 0.02, size=(n, 3)).astype(dtype)
    idx = np.sort(rng.uniform(lo, lo + 1.3, size=n))
    plain = LieIncrementStream.from_increments(inc, indices=idx, width=3, depth=4, resolution=res)
    plain.auto_range_table = False
    table = LieIncrementStream.from_increments(inc, indices=idx, width=3, depth=4, resolution=res)
    table.build_range_table()
    assert table._tree.range_table and table._tree.rows == plain._build_tree().rows
    q = np.sort(rng.uniform(lo - 0.2, lo + 1.5, size=(700, 2)), axis=1)
    grid = np.ldexp(1.0, -res)
    q[:100] = np.round(q[:100] / grid) * grid            # leaf-aligned ends
    q[100:150, 1] = q[100:150, 0] + 3 * grid              # inside one block
    q[150:160, 1] = q[150:160, 0]                          # empty
    q[160:170] = [lo + 5.0, lo + 6.0]                      # outside the support
    tol = 1e-12 if dtype == np.float64 else 1e-6
    for resolution in (None, res + 3):
        a = plain.log_signature_batch(q[:, 0], q[:, 1], resolution=resolution).cpu().numpy()
        b = table.log_signature_batch(q[:, 0], q[:, 1], resolution=resolution).cpu().numpy()
        scale = np.maximum(np.abs(a).max(axis=1, keepdims=True), 1e-300)
        assert float((np.abs(a - b) / scale).max()) <= tol, resolution
        sa = plain.signature_batch(q[:, 0], q[:, 1], resolution=resolution).cpu().numpy()
        sb = table.signature_batch(q[:, 0], q[:, 1], resolution=resolution).cpu().numpy()
        assert level_rel_err(sb, sa, 3, 4) <= tol
