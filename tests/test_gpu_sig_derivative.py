"""Forward-mode signature derivative (rpyb_sig_derivative, the reference's
Context::sig_derivative / Stream::signature_derivative) on the GPU, against:
the reference test suite's known answers
(tests/streams/test_lie_increment_path.py:219-263), central finite differences
of exp for single pairs, and the oracle restatement of
algebra/src/lite_context.h:577-636 for lists of several pairs.

Tolerances: known answers 1e-14 absolute; finite differences (h = 1e-5)
1e-8 relative to the largest entry; float64 lists 1e-12 and float32 lists
2e-6 per-level relative against the restatement."""
import numpy as np
import pytest
import torch

from roughpy_b200 import compute as rpc
from roughpy_b200.streams import (LieIncrementStream, RealInterval, sig_derivative,
                                  sig_derivative_batch)
from tests._util import level_rel_err
from tests.test_streams_host import arith

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("depth,expected", [
    (1, [0.0, 0.0, 1.0, 0.0]),
    (2, [0.0, 0.0, 1.0, 0.0, 0.0, 0.1, 0.0, 0.1, 0.4, 0.3, 0.0, 0.3, 0.0]),
])
def test_reference_known_answers(depth, expected):
    p = LieIncrementStream.from_increments(np.array([[0.2, 0.4, 0.6]]), indices=np.array([0.0]),
                                           width=3, depth=depth)
    d = p.signature_derivative(RealInterval(0.0, 1.0), np.array([0.0, 1.0, 0.0]))
    assert np.max(np.abs(d - np.array(expected))) <= 1e-14
    # the list form with one pair gives the same
    d2 = p.signature_derivative([(RealInterval(0.0, 1.0), np.array([0.0, 1.0, 0.0]))])
    assert np.array_equal(d, d2)


@pytest.mark.parametrize("w,d", [(3, 4), (2, 6), (4, 3)])
def test_single_pair_is_the_derivative_of_exp(w, d):
    rng = np.random.default_rng(w * 10 + d)
    lb, tb = rpc.LieBasis(w, d), rpc.TensorBasis(w, d)
    L, T = lb.size(), tb.size()
    x = rng.normal(0, 0.5, L)
    p = rng.normal(0, 1.0, L)
    got = sig_derivative([(x, p)], w, d)

    def sig(lie):
        t = torch.zeros((1, T), dtype=torch.float64, device="cuda")
        rpc._internals.dense_lie_to_tensor(t, torch.from_numpy(lie[None]).cuda(),
                                           lb.get_l2t_matrix(), lb, tb)
        e = torch.zeros_like(t)
        rpc._internals.dense_ft_exp(e, t, tb)
        return e[0].cpu().numpy()
    h = 1e-5
    fd = (sig(x + h * p) - sig(x - h * p)) / (2 * h)
    assert np.max(np.abs(got - fd)) <= 1e-8 * max(1.0, np.max(np.abs(fd)))


@pytest.mark.parametrize("w,d", [(3, 3), (2, 4), (4, 3)])
def test_lists_against_restatement(golden, w, d):
    a = arith(golden, w, d)
    rng = np.random.default_rng(100 + w * d)
    lens = [3, 1, 0, 5]
    off = np.concatenate([[0], np.cumsum(lens)])
    n = int(off[-1])
    lg = rng.normal(0, 0.4, (n, a.L))
    pt = rng.normal(0, 1.0, (n, a.L))
    want = np.stack([a.sig_derivative(list(zip(lg[off[q]:off[q + 1]], pt[off[q]:off[q + 1]])))
                     for q in range(len(lens))])
    got = sig_derivative_batch(lg, pt, off, w, d).cpu().numpy()
    assert level_rel_err(got, want, w, d) <= 1e-12
    got32 = sig_derivative_batch(lg.astype(np.float32), pt.astype(np.float32), off, w, d)
    assert got32.dtype == torch.float32
    assert level_rel_err(got32.double().cpu().numpy(), want, w, d) <= 2e-6


def test_stream_list_form_matches_restatement_of_its_log_signatures(golden):
    w, d = 3, 3
    a = arith(golden, w, d)
    rng = np.random.default_rng(7)
    inc = rng.normal(0, 0.3, (40, w))
    idx = np.sort(rng.uniform(0, 1, 40))
    st = LieIncrementStream.from_increments(inc, indices=idx, width=w, depth=d, resolution=5)
    ivs = [(0.1, 0.45), (0.3, 0.9), (0.0, 0.2)]
    perts = [rng.normal(size=a.L) for _ in ivs]
    got = st.signature_derivative([((x, y), p) for (x, y), p in zip(ivs, perts)])
    lies = [st.log_signature(x, y) for x, y in ivs]
    want = a.sig_derivative(list(zip(lies, perts)))
    assert level_rel_err(got, want, w, d) <= 1e-12
