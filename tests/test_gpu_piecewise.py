"""PiecewiseAbelianStream queries (rpyb_piecewise_query) against the oracle
restatement of the reference's piecewise abelian stream and stream query path,
and the reference test suite's full-data identity
(tests/streams/test_piecewise_lie_path.py:41-51).

Tolerances: log-signatures 1e-12 absolute (scaled by the largest entry),
signatures 1e-12 per-level relative."""
import numpy as np
import pytest

from oracle import streams_ref as R
from roughpy_b200.streams import PiecewiseAbelianStream, RealInterval
from tests._util import level_rel_err
from tests.test_streams_host import arith

pytestmark = pytest.mark.gpu


def close(got, want, tol=1e-12):
    scale = max(1.0, float(np.max(np.abs(want))))
    assert float(np.max(np.abs(np.asarray(got) - want))) <= tol * scale


@pytest.mark.parametrize("count", [1, 2, 5])
def test_full_data_log_signature_is_cbh_of_the_pieces(golden, count):
    a = arith(golden, 4, 3)
    rng = np.random.default_rng(count)
    data = []
    for i in range(count):
        v = np.zeros(a.L)
        v[:4] = rng.normal(0.0, 1.0, 4)
        data.append((RealInterval(float(i), float(i + 1)), v))
    st = PiecewiseAbelianStream.construct(data, width=4, depth=3)
    close(st.log_signature(5), a.cbh([v for _, v in data]))


@pytest.mark.parametrize("w,d", [(3, 3), (2, 4), (4, 3)])
def test_random_pieces_against_restatement(golden, w, d):
    a = arith(golden, w, d)
    rng = np.random.default_rng(w * 31 + d)
    # pieces of uneven length with a gap, Lie elements with bracket terms
    edges = np.cumsum(rng.uniform(0.05, 0.4, 12)) - 0.6
    pieces = []
    for i in range(11):
        if i == 6:
            continue
        pieces.append((float(edges[i]), float(edges[i + 1]), rng.normal(0, 0.5, a.L)))
    ref = R.PiecewiseRef(a, pieces)
    st = PiecewiseAbelianStream.construct([((p, q), v) for p, q, v in pieces], width=w, depth=d)
    qs = np.sort(rng.uniform(edges[0] - 0.2, edges[-1] + 0.2, (20, 2)), axis=1)
    got = st.log_signature_batch(qs[:, 0], qs[:, 1]).cpu().numpy()
    want = np.stack([ref.log_signature(x, y) for x, y in qs])
    close(got, want)
    sig = st.signature_batch(qs[:, 0], qs[:, 1]).cpu().numpy()
    assert level_rel_err(sig, np.stack([ref.signature(x, y) for x, y in qs]), w, d) <= 1e-12
    for res in (1, 4):
        got = st.log_signature_batch(qs[:6, 0], qs[:6, 1], resolution=res).cpu().numpy()
        close(got, np.stack([ref.log_signature(x, y, res) for x, y in qs[:6]]))
    # single-query forms and the reference's argument rules
    close(st.log_signature(float(qs[3, 0]), float(qs[3, 1])), want[3])
    close(st.log_signature(3), ref.log_signature(resolution=3))
    with pytest.raises(TypeError):
        st.log_signature(0.5)
