"""Stream.restrict and Stream.simplify (streams/src/stream.cpp:73-89 and
:232-258) on the GPU streams: a restricted stream's queries are those of the
restatement with the support replaced; a simplified stream's pieces are the
original log-signatures over the partition's intervals.

Tolerances as for the other streams: log-signatures within 1e-12 of the
larger of 1 and the largest coordinate."""
import numpy as np
import pytest

from oracle import streams_ref as R
from roughpy_b200.streams import (LieIncrementStream, Partition, PiecewiseAbelianStream,
                                  RealInterval)

pytestmark = pytest.mark.gpu


def _arith(golden, w, d):
    from tests.test_streams_host import arith
    return arith(golden, w, d)


def lie_close(got, want, tol):
    scale = max(1.0, float(np.max(np.abs(want))))
    assert float(np.max(np.abs(np.asarray(got) - want))) <= tol * scale


def _stream():
    rng = np.random.default_rng(21)
    inc = rng.normal(0, 0.2, (200, 3))
    idx = np.sort(rng.uniform(0.0, 1.0, 200))
    return inc, idx, LieIncrementStream.from_increments(inc, indices=idx, width=3, depth=3,
                                                        resolution=8)


def test_restrict_trims_queries_to_the_new_support(golden):
    inc, idx, st = _stream()
    r = st.restrict(RealInterval(0.25, 0.75))
    lie_close(r.log_signature(RealInterval(0.0, 1.0)), st.log_signature(RealInterval(0.25, 0.75)),
              1e-13)
    ref = R.StreamRef(_arith(golden, 3, 3), inc, idx, 8)
    ref.support = (0.25, 0.75)
    rng = np.random.default_rng(22)
    qs = np.sort(rng.uniform(-0.2, 1.2, (15, 2)), axis=1)
    got = r.log_signature_batch(qs[:, 0], qs[:, 1]).cpu().numpy()
    lie_close(got, np.stack([ref.log_signature(a, b) for a, b in qs]), 1e-12)
    # a support wider than the original one: the events stay what they are
    w = st.restrict(RealInterval(-1.0, 2.0))
    lie_close(w.log_signature(RealInterval(-1.0, 2.0), 8), st.log_signature(RealInterval(0.0, 1.0), 8),
              1e-12)


def test_simplify_gives_the_pieces_log_signatures():
    _, idx, st = _stream()
    part = Partition(RealInterval(0.0, 1.0), [0.25, 0.5, 0.75])
    pw = st.simplify(part, resolution=8)
    assert isinstance(pw, PiecewiseAbelianStream)
    assert pw.resolution == 8 and (pw.support.inf, pw.support.sup) == (st.support.inf, st.support.sup)
    for i in range(len(part)):
        lie_close(pw.log_signature(part[i], resolution=2), st.log_signature(part[i], resolution=8),
                  1e-12)
    # two adjacent pieces combine by CBH into the original over their union
    lie_close(pw.log_signature(RealInterval(0.0, 0.5), resolution=1),
              st.log_signature(RealInterval(0.0, 0.5), resolution=8), 1e-12)
    # a lower depth truncates the pieces
    pw2 = st.simplify(part, resolution=8, depth=2)
    assert pw2.depth == 2
    L2 = pw2.lie_basis.size()
    lie_close(pw2.log_signature(part[2], resolution=2), st.log_signature(part[2], resolution=8)[:L2],
              1e-12)
