"""Hall basis and Lie <-> tensor maps built on the host by librpyb.so,
checked against the reference's roughpy.compute outputs (tests/golden)."""
import numpy as np
import pytest

from roughpy_b200 import compute as rpc

SHAPES = [(2, 4), (3, 4), (4, 5), (6, 5), (8, 5), (5, 4)]


def csr_apply(m, x):
    x = np.atleast_2d(x)
    out = np.zeros((x.shape[0], m.shape[0]))
    for r in range(m.shape[0]):
        s, e = m.indptr[r], m.indptr[r + 1]
        out[:, r] = x[:, m.indices[s:e]] @ m.data[s:e]
    return out


@pytest.mark.parametrize("w,d", SHAPES)
def test_hall_basis_matches_reference(golden, w, d):
    g = golden["lie_maps"]
    lb = rpc.LieBasis(w, d)
    np.testing.assert_array_equal(lb.data, g[f"w{w}d{d}_data"])
    np.testing.assert_array_equal(lb.degree_begin, g[f"w{w}d{d}_degree_begin"])
    assert rpc.check_lie_basis_data(w, d, g[f"w{w}d{d}_data"])


@pytest.mark.parametrize("w,d", SHAPES)
def test_maps_match_reference_on_random_vectors(golden, w, d):
    g = golden["lie_maps"]
    t = f"w{w}d{d}"
    lb = rpc.LieBasis(w, d)
    l2t = lb.get_l2t_matrix(np.float64)
    t2l = lb.get_t2l_matrix(np.float64)
    np.testing.assert_allclose(csr_apply(l2t, g[f"{t}_l2t_in"]), g[f"{t}_l2t_out"],
                               rtol=0, atol=1e-12)
    np.testing.assert_allclose(csr_apply(t2l, g[f"{t}_t2l_in"]), g[f"{t}_t2l_out"],
                               rtol=0, atol=1e-12)


@pytest.mark.parametrize("w,d", [(2, 4), (3, 3), (4, 3)])
def test_maps_equal_reference_exactly(golden, w, d):
    g = golden["lie_maps"]
    lb = rpc.LieBasis(w, d)
    np.testing.assert_array_equal(lb.get_l2t_matrix().todense(), g[f"w{w}d{d}_l2t_dense"])
    np.testing.assert_array_equal(lb.get_t2l_matrix().todense(), g[f"w{w}d{d}_t2l_dense"])


def test_t2l_inverts_l2t_on_lie_elements():
    # tests/compute/test_l2t_and_t2l.py:8-56 (round trip at decimal=15)
    lb = rpc.LieBasis(3, 4)
    rng = np.random.default_rng(5)
    x = rng.standard_normal((4, lb.size()))
    back = csr_apply(lb.get_t2l_matrix(), csr_apply(lb.get_l2t_matrix(), x))
    np.testing.assert_array_almost_equal(back, x, decimal=15)


def test_lie_basis_value_semantics():
    """As the reference's LieBasis type (tests/compute/test_lie_basis.py:24-140):
    equal shape means equal bases and equal hashes, usable as set members and
    dict keys; a different width or depth differs."""
    from roughpy_b200 import compute as rpc
    a, b = rpc.LieBasis(3, 4), rpc.LieBasis(3, 4)
    c, d = rpc.LieBasis(4, 4), rpc.LieBasis(3, 5)
    assert a == b and hash(a) == hash(b) and not (a != b)
    assert a != c and a != d and c != d
    assert len({a, b, c}) == 2
    assert len({hash(rpc.LieBasis(2, 3)), hash(rpc.LieBasis(3, 2)), hash(rpc.LieBasis(4, 5))}) == 3
    assert (a == 3) is False
