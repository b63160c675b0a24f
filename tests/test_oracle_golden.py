"""The CPU oracle (C restatement) against the reference's own outputs.

The fixtures in tests/golden were produced by RoughPy's compiled
roughpy.compute extension; the known answers restate the reference's
tests/compute suite.  No GPU is needed.
"""
import numpy as np
import pytest

import oracle
from tests._util import level_rel_err

CASES = [(2, 4), (3, 3), (4, 3), (2, 6), (5, 2)]
TOL = 1e-13


def test_known_answer_fma_explicit(golden):
    # tests/compute/test_ft_fma.py:7-20
    g = golden["tensor_ops"]
    got = oracle.ft_fma(2, 2, np.zeros(7), g["fma_explicit_b"], g["fma_explicit_c"])
    np.testing.assert_array_equal(got, [-2, 7, -3, 5.5, 3, 10, 4])
    np.testing.assert_array_equal(g["fma_explicit_out"], [-2, 7, -3, 5.5, 3, 10, 4])


def test_known_answer_exp_letter_and_log_identity():
    # tests/compute/test_exp_and_log.py:13-49
    np.testing.assert_array_equal(oracle.ft_exp(2, 2, np.zeros(7)), [1, 0, 0, 0, 0, 0, 0])
    np.testing.assert_array_equal(oracle.ft_exp(2, 2, np.array([0, 1.0, 0, 0, 0, 0, 0])),
                                  [1, 1, 0, 0.5, 0, 0, 0])
    np.testing.assert_array_equal(oracle.ft_log(2, 2, np.array([1.0, 0, 0, 0, 0, 0, 0])),
                                  np.zeros(7))


@pytest.mark.parametrize("w,d", CASES)
def test_fma_bounds(golden, w, d):
    g = golden["tensor_ops"]
    t = f"w{w}d{d}"
    A, B, C = g[f"{t}_A"], g[f"{t}_B"], g[f"{t}_C"]
    for (od, ld, rd) in [(-1, -1, -1), (d - 1, -1, -1), (-1, d - 1, -1), (-1, -1, 1), (2, 1, 1)]:
        got = oracle.ft_fma(w, d, A, B, C, bounds=(0, od, 0, ld, 0, rd))
        assert level_rel_err(got, g[f"{t}_fma_{od}_{ld}_{rd}"], w, d) <= TOL


@pytest.mark.parametrize("w,d", CASES)
def test_inplace_mul(golden, w, d):
    g = golden["tensor_ops"]
    t = f"w{w}d{d}"
    for (od, rd) in [(-1, -1), (-1, 1), (d - 1, -1)]:
        got = oracle.ft_inplace_mul(w, d, g[f"{t}_B"], g[f"{t}_C"], bounds=(0, od, 0, rd))
        assert level_rel_err(got, g[f"{t}_imul_{od}_{rd}"], w, d) <= TOL


@pytest.mark.parametrize("w,d", CASES)
def test_series(golden, w, d):
    g = golden["tensor_ops"]
    t = f"w{w}d{d}"
    X, A = g[f"{t}_X"], g[f"{t}_A"]
    assert level_rel_err(oracle.ft_exp(w, d, X), g[f"{t}_exp"], w, d) <= TOL
    assert level_rel_err(oracle.ft_fmexp(w, d, A, X), g[f"{t}_fmexp"], w, d) <= TOL
    assert level_rel_err(oracle.ft_log(w, d, g[f"{t}_exp"]), g[f"{t}_log"], w, d) <= 1e-12
    assert level_rel_err(oracle.ft_log(w, d, A), g[f"{t}_log_A"], w, d) <= 1e-12
    assert level_rel_err(oracle.antipode(w, d, A), g[f"{t}_antipode"], w, d) == 0.0
    got = oracle.adjoint_left_mul(w, d, g[f"{t}_B"], g[f"{t}_C"], d, d, d)
    assert level_rel_err(got, g[f"{t}_adjlmul"], w, d) <= TOL


def test_signatures(golden):
    g = golden["signatures"]
    for key in g.files:
        if not key.endswith("_sig"):
            continue
        t = key[:-4]
        w, d = int(t[1:t.index("d")]), int(t[t.index("d") + 1:])
        got = oracle.signatures(w, d, g[f"{t}_inc"], g[f"{t}_offsets"])
        assert level_rel_err(got, g[key], w, d) <= 1e-13, t


def test_antipode_is_group_inverse():
    # tests/compute/test_antipode.py:10-37, restated on the oracle
    rng = np.random.default_rng(1234)
    w, d = 4, 3
    x = np.zeros(oracle.tensor_size(w, d))
    x[1:1 + w] = rng.normal(size=w)
    sig = oracle.ft_exp(w, d, x)
    prod = oracle.ft_mul(w, d, oracle.antipode(w, d, sig), sig)
    expect = np.zeros_like(sig)
    expect[0] = 1.0
    np.testing.assert_allclose(prod, expect, atol=1e-14)
