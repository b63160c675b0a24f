"""Restatement of RoughPy's stream query path -- TEST INFRASTRUCTURE ONLY.

Mirrors, step for step and in float64:
  roughpy/src/streams/lie_increment_stream.cpp:73-246  (from_increments: indices,
      resolution heuristic, support)
  streams/src/lie_increment_stream.cpp:116-199         (events keyed by time, first
      wins; leaf log-signature = cbh of the events in [inf, sup))
  streams/src/dyadic_caching_layer.cpp:86-154          (cache at the stream resolution,
      recursive halves above it, expand-or-zero below it)
  streams/src/stream.cpp:37-171                        (trim to support, resolution,
      dissection, cbh of the pieces, signature = exp(l2t(.)))
  algebra/src/context.cpp:156-215                      (cbh = log of the fmexp chain,
      then t2l; one element is returned as is)
  intervals/src/dyadic_interval.cpp:191-224            (dissection, pure Python here)

The tensor arithmetic is injected (`Arith`): the C oracle by default, or the
reference's own roughpy.compute when generating golden fixtures.  The Lie maps
are dense matrices supplied by the caller (pinned to the reference in
tests/golden/lie_maps.npz).
"""
from __future__ import annotations

import bisect
import math

import numpy as np


# ------------------------------------------------------------ dyadic intervals
def _mod(a, b):
    r = a % b  # Python % is already non-negative for b > 0
    return r


def _rebase(k, p, res):
    if k == 0:
        return 0, res, True
    if res >= p:
        return k * (1 << (res - p)), res, True
    r = p - res
    while k % (1 << r) != 0:
        r -= 1
    return k // (1 << r), p - r, res == p - r


def _from_dyadic(k, p, res):
    """clopen DyadicInterval(Dyadic(k, p), res)"""
    k2, p2, ok = _rebase(k, p, res)
    if not ok:
        pw = 1 << (p - res)
        k2 = k - _mod(k, pw)
        k2, p2, _ = _rebase(k2, p, res)
    return k2, p2


def _contains(bk, bp, ek, ep):
    if ep >= bp:
        pw = 1 << (ep - bp)
        return bk * pw == ek - _mod(ek, pw)
    return False


def _aligned(k, p):
    pk, pp = _from_dyadic(k, p, p - 1)
    bk, bp = _from_dyadic(pk, pp, p)
    return (bk, bp) == (k, p) or math.ldexp(bk, -bp) == math.ldexp(k, -p)


def to_dyadic_intervals(inf, sup, tol):
    """Clopen dissection; returns [(k, p)] in order."""
    bk, bp = math.floor(math.ldexp(inf, tol)), tol
    ek, ep = math.floor(math.ldexp(sup, tol)), tol
    front, back = [], []
    while not _contains(bk, bp, ek, ep):
        nk, np_ = _from_dyadic(bk, bp, bp - 1)
        if not _aligned(bk, bp):
            ck, cp = _from_dyadic(nk, np_, np_ + 1)       # shrink to contained end
            ck = ck + 1 if ck % 2 == 0 else ck - 1         # flip -> omitted end
            front.append((ck, cp))
            nk += 1
        bk, bp = nk, np_
    nk, np_ = ek, ep
    while True:
        nk, np_ = _from_dyadic(nk, np_, np_ - 1)
        if not _contains(bk, bp, nk, np_):
            break
        if not _aligned(ek, ep):
            back.append(_from_dyadic(nk, np_, np_ + 1))
        ek, ep = nk, np_
    return front + back[::-1]


def param_to_resolution(accuracy):
    _, e = math.frexp(accuracy)
    return -min(5, e - 1)


def stream_param_to_resolution(length):
    _, e = math.frexp(length)
    return -min(0, e - 1)


# ------------------------------------------------------------ arithmetic
class Arith:
    """Dense float64 tensor arithmetic used by the restatement."""

    def __init__(self, width, depth, l2t, t2l, exp, fmexp, log, mul=None):
        self.width, self.depth = width, depth
        self.l2t = np.asarray(l2t, dtype=np.float64)   # [tensor, lie]
        self.t2l = np.asarray(t2l, dtype=np.float64)   # [lie, tensor]
        self.exp, self.fmexp, self.log, self.mul = exp, fmexp, log, mul
        self.T = self.l2t.shape[0]
        self.L = self.l2t.shape[1]

    @classmethod
    def from_oracle(cls, width, depth, l2t, t2l):
        import oracle
        return cls(width, depth, l2t, t2l,
                   lambda x: oracle.ft_exp(width, depth, x),
                   lambda a, x: oracle.ft_fmexp(width, depth, a, x),
                   lambda x: oracle.ft_log(width, depth, x),
                   lambda a, b: oracle.ft_mul(width, depth, a, b))

    def cbh(self, lies):
        # context.cpp:187-208
        if len(lies) == 1:
            return lies[0].copy()
        coll = np.zeros(self.T)
        coll[0] = 1.0
        for lie in lies:
            if np.any(lie != 0):
                coll = self.fmexp(coll, self.l2t @ lie)
        return self.t2l @ self.log(coll)

    def to_signature(self, lie):
        return self.exp(self.l2t @ lie)

    def sig_derivative(self, pairs):
        """algebra/src/lite_context.h:577-636 (sig_derivative_impl with
        derive_series_compute and sig_derivative_single), for a list of
        (log-signature, perturbation) Lie coordinate pairs."""
        result = np.zeros(self.T)
        for lie, pert in pairs:
            x = self.l2t @ np.asarray(lie, dtype=np.float64)
            p = self.l2t @ np.asarray(pert, dtype=np.float64)
            sig = self.exp(x)
            series = p.copy()
            factor = 1.0
            ad = self.mul(x, p) - self.mul(p, x)
            for d in range(1, self.depth + 1):
                factor *= d + 1
                series = series + ad / factor if d % 2 == 0 else series - ad / factor
                ad = self.mul(x, ad) - self.mul(ad, x)
            result = self.mul(result, sig) + self.mul(sig, series)
        return result


class StreamRef:
    """LieIncrementStream + DyadicCachingLayer + Stream, restated."""

    def __init__(self, arith, data, indices=None, resolution=None):
        self.a = arith
        rows = np.asarray(data, dtype=np.float64)
        if rows.ndim == 1:
            rows = rows.reshape(1, -1)
        n = rows.shape[0]
        lies = np.zeros((n, arith.L))
        c = min(rows.shape[1], arith.L)
        lies[:, :c] = rows[:, :c]
        if indices is None:
            idx = [float(i) for i in range(n)]
            res = 0 if resolution is None else resolution
        else:
            idx = [float(v) for v in indices]
            if resolution is None:
                min_diff = math.inf
                res = 0
                for v in idx:
                    min_diff = min(min_diff, v - 0.0)
                    res = param_to_resolution(min_diff) + 1
            else:
                res = resolution
        self.resolution = res
        self.data = {}
        for t, lie in zip(idx, lies):
            if t not in self.data:          # try_emplace: the first one wins
                self.data[t] = lie
        self.keys = sorted(self.data)
        self.support = (min(idx), max(idx) + math.ldexp(1.0, -res))
        self.cache = {}

    def _leaf_events(self, inf, sup):
        lo = bisect.bisect_left(self.keys, inf)
        hi = bisect.bisect_left(self.keys, sup)
        return [self.data[t] for t in self.keys[lo:hi]]

    def _dyadic_logsig(self, k, p):
        R = self.resolution
        if p == R:
            key = (k, p)
            if key not in self.cache:
                lies = self._leaf_events(math.ldexp(k, -p), math.ldexp(k + 1, -p))
                self.cache[key] = (np.zeros(self.a.L) if not lies else self.a.cbh(lies))
            return self.cache[key]
        if p > R:
            tk, tp = _from_dyadic(k, p, R)
            # rational_equals on the included ends
            if math.ldexp(tk, -tp) == math.ldexp(k, -p):
                return self._dyadic_logsig(tk, tp)
            return np.zeros(self.a.L)
        lhs = self._dyadic_logsig(2 * k, p + 1)
        rhs = self._dyadic_logsig(2 * k + 1, p + 1)
        if not np.any(lhs):
            return rhs
        if not np.any(rhs):
            return lhs
        return self.a.cbh([lhs, rhs])

    def log_signature(self, inf=None, sup=None, resolution=None):
        s0, s1 = self.support
        if inf is None:
            inf, sup = s0, s1
        if sup < s0 or inf > s1:
            return np.zeros(self.a.L)
        inf, sup = max(inf, s0), min(sup, s1)
        length = sup - inf
        if length == 0.0:
            return np.zeros(self.a.L)
        res = max(self.resolution, stream_param_to_resolution(length) + 2) \
            if resolution is None else resolution
        pieces = [self._dyadic_logsig(k, p) for (k, p) in to_dyadic_intervals(inf, sup, res)]
        pieces = [x for x in pieces if np.any(x)]
        if not pieces:
            return np.zeros(self.a.L)
        return self.a.cbh(pieces)

    def signature(self, inf=None, sup=None, resolution=None):
        return self.a.to_signature(self.log_signature(inf, sup, resolution))


class PiecewiseRef:
    """PiecewiseAbelianStream + Stream queries, restated
    (streams/src/piecewise_abelian_stream.cpp:154-189 through
    streams/src/stream_base.cpp:81-96 and streams/src/stream.cpp:37-171; the
    Python constructor's support and resolution,
    roughpy/src/streams/piecewise_abelian_stream.cpp:51-95)."""

    def __init__(self, arith, pieces, resolution=None):
        # pieces: [(inf, sup, lie coordinates)] in order
        self.a = arith
        self.pieces = [(float(p), float(q), np.asarray(v, dtype=np.float64)) for p, q, v in pieces]
        self.support = (min(p for p, _, _ in self.pieces), max(q for _, q, _ in self.pieces))
        self.resolution = 0 if resolution is None else int(resolution)

    def _dyadic_logsig(self, k, p):
        a, b = math.ldexp(k, -p), math.ldexp(k + 1, -p)
        lies = []
        for pa, pb, lie in self.pieces:
            if pa >= b:
                break
            if pb <= a:
                continue
            if pa >= a and pb <= b:
                lies.append(lie)
            else:
                # the reference's branch condition `pb <= pb` always holds, so
                # every partial overlap takes to_multiplier_upper(piece, a)
                lies.append(lie * ((pb - a) / (pb - pa)))
        if not lies:
            return np.zeros(self.a.L)
        return self.a.cbh(lies)

    log_signature = StreamRef.log_signature

    def signature(self, inf=None, sup=None, resolution=None):
        return self.a.to_signature(self.log_signature(inf, sup, resolution))


class TickRef:
    """TickStream restated (streams/src/tick_stream.cpp:41-201 with
    streams/include/roughpy/streams/tick_stream.h:66-83), queried through the
    Stream rules (streams/src/stream.cpp:37-171, stream_base.cpp:81-96).
    Clopen intervals.

    Events (time, Lie coordinates) are keyed by their dyadic interval at the
    stream resolution; events sharing one are combined by CBH in input order.
    The cache holds, for the sub-intervals visited by the recursion from the
    smallest dyadic intervals containing all negative and all positive events,
    the CBH of the two halves; a dyadic query piece takes the cached value of
    the smallest dyadic interval containing the events inside it."""

    def __init__(self, arith, events, resolution=0, support=(0.0, 1.0)):
        self.a = arith
        self.resolution = int(resolution)
        self.support = (float(support[0]), float(support[1]))
        R = self.resolution
        self.data = {}
        index = set()
        for t, lie in events:
            k = math.floor(math.ldexp(float(t), R))
            lie = np.asarray(lie, dtype=np.float64)
            full = np.zeros(arith.L)
            full[:lie.shape[0]] = lie
            if (k, R) in self.data:
                self.data[(k, R)] = arith.cbh([self.data[(k, R)], full])
            else:
                self.data[(k, R)] = full
            index.add(math.ldexp(k, -R))
        self.granular = sorted(index)
        # tick_stream.cpp:60-98: the negative events are those at or before
        # 0, the positive ones those from the first leaf start >= 0 (a clopen
        # leaf at 0 ends above 0), so the leaf at 0 belongs to both
        neg = self._smallest_of_range(0, bisect.bisect_right(self.granular, 0.0))
        pos = self._smallest_of_range(bisect.bisect_left(self.granular, 0.0),
                                      len(self.granular))
        for root in (neg, pos):
            if root is not None:
                self._recursive(root)

    def _leaf(self, t):
        R = self.resolution
        return (math.floor(math.ldexp(t, R)), R)

    def _smallest_of_range(self, lo, hi):
        # tick_stream.cpp:41-98: expand the first event's leaf until it
        # contains the last event's leaf
        if hi <= lo:
            return None
        k, p = self._leaf(self.granular[lo])
        ek, ep = self._leaf(self.granular[hi - 1])
        steps = 0
        while not _contains(k, p, ek, ep):
            k, p = _from_dyadic(k, p, p - 1)
            steps += 1
            if steps > 4 * 64:
                # a range from before 0 to the leaf at 0: k stays -1 and the
                # reference's loop does not end
                raise ValueError("no dyadic interval contains events on both sides of 0")
        return (k, p)

    def _smallest(self, k, p):
        inf, sup = math.ldexp(k, -p), math.ldexp(k + 1, -p)
        lo = bisect.bisect_left(self.granular, inf)
        hi = bisect.bisect_left(self.granular, sup)
        return self._smallest_of_range(lo, hi)

    def _recursive(self, di):
        # tick_stream.cpp:100-123
        s = self._smallest(*di)
        if s is None:
            return np.zeros(self.a.L)
        it = self.data.get(s)
        if it is not None and np.any(it):
            return it
        if s[1] == self.resolution:
            self.data.setdefault(s, np.zeros(self.a.L))
            return self.data[s]
        left = self._recursive((2 * s[0], s[1] + 1))
        right = self._recursive((2 * s[0] + 1, s[1] + 1))
        self.data[s] = self.a.cbh([left, right])
        return self.data[s]

    def _dyadic_logsig(self, k, p):
        # tick_stream.cpp:188-201 (log_signature_impl)
        s = self._smallest(k, p)
        if s is None:
            return np.zeros(self.a.L)
        return self.data[s]

    log_signature = StreamRef.log_signature

    def signature(self, inf=None, sup=None, resolution=None):
        return self.a.to_signature(self.log_signature(inf, sup, resolution))
