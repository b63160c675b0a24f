"""GPU tick streams (roughpy_b200.streams.TickStream) against the restated
TickStream (oracle/streams_ref.py TickRef: the reference's compressed dyadic
recursion, keyed by the smallest dyadic interval holding a query piece's
events) and the reference test suite's known answer.

Tolerances as for the other streams: log-signatures within 1e-11 of the
larger of 1 and the largest coordinate."""
import numpy as np
import pytest

from oracle import streams_ref as R
from roughpy_b200.streams import RealInterval, TickStream

pytestmark = pytest.mark.gpu


def _arith(golden, w, d):
    from tests.test_streams_host import arith
    return arith(golden, w, d)


def lie_close(got, want, tol):
    scale = max(1.0, float(np.max(np.abs(want))))
    assert float(np.max(np.abs(np.asarray(got) - want))) <= tol * scale


def test_two_ticks_at_one_time_known_answer():
    """tests/streams/test_tick_stream.py:107-115: increments "first" then
    "second" at t = 1 give Lie([1, 1, 0.5]) at width 2, depth 2; the reverse
    input order flips the bracket (events of one interval are combined in
    input order, not by time)."""
    e = np.eye(2)
    st = TickStream.from_lie_events([1.0, 1.0], e, 2, 2, support=(0.0, 2.0))
    np.testing.assert_allclose(st.log_signature(RealInterval(0.0, 2.0), 2), [1.0, 1.0, 0.5],
                               atol=1e-15)
    st = TickStream.from_lie_events([1.0, 1.0], e[::-1], 2, 2, support=(0.0, 2.0))
    np.testing.assert_allclose(st.log_signature(RealInterval(0.0, 2.0), 2), [1.0, 1.0, -0.5],
                               atol=1e-15)


@pytest.mark.parametrize("w,d,res,lie_rows", [(2, 4, 5, False), (3, 3, 4, True),
                                              (4, 3, 6, False)])
def test_random_ticks_against_restatement(golden, w, d, res, lie_rows):
    """Unsorted times with several events per interval, negative times,
    increments or full Hall coordinates; queries inside and across the
    support at the automatic, a coarser and a finer resolution."""
    a = _arith(golden, w, d)
    rng = np.random.default_rng(w * 10 + d + res)
    n = 60
    cand = np.concatenate([np.arange(-25, 0), np.arange(1, 50)])   # no tick at 0 next to t < 0
    leaves = rng.choice(cand, size=n)
    times = (leaves + rng.uniform(0, 1, n)) / 2.0 ** res   # several ticks share intervals
    cols = a.L if lie_rows else w
    rows = rng.normal(0, 0.3, (n, cols))
    support = (float(times.min()) - 0.1, float(times.max()) + 0.2)
    ref = R.TickRef(a, list(zip(times, rows)), resolution=res, support=support)
    st = TickStream.from_lie_events(times, rows, w, d, resolution=res, support=support)
    qs = np.sort(rng.uniform(support[0] - 0.3, support[1] + 0.3, size=(20, 2)), axis=1)
    for q_res in (None, res - 2, res + 2):
        got = st.log_signature_batch(qs[:, 0], qs[:, 1], resolution=q_res).cpu().numpy()
        want = np.stack([ref.log_signature(lo, hi, q_res) for lo, hi in qs])
        lie_close(got, want, 1e-11)
    # the whole support, and the signature as exp(l2t(log-signature))
    lie_close(st.log_signature(), ref.log_signature(), 1e-11)
    sig = st.signature_batch(qs[:5, 0], qs[:5, 1]).cpu().numpy()
    want = np.stack([ref.signature(lo, hi) for lo, hi in qs[:5]])
    lie_close(sig, want, 1e-11)


def test_default_support_trims_queries():
    """Without a support the stream covers [0, 1), as the reference's
    tick-stream constructor defaults it: ticks outside are not seen."""
    st = TickStream.from_lie_events([0.25, 1.5], np.eye(2), 2, 2)
    got = st.log_signature(RealInterval(0.0, 2.0), 1)
    np.testing.assert_allclose(got, [1.0, 0.0, 0.0], atol=1e-15)
