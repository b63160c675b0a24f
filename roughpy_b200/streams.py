"""GPU streams with dyadic caching: a drop-in for RoughPy's ``LieIncrementStream``.

``LieIncrementStream.from_increments(data, ...)`` builds a stream of Lie
increments keyed by time, as RoughPy does
(roughpy/src/streams/lie_increment_stream.cpp:73-246, streams/src/
lie_increment_stream.cpp:116-199).  ``signature`` / ``log_signature`` answer
interval queries with the reference's semantics (streams/src/stream.cpp:54-171,
streams/src/dyadic_caching_layer.cpp:86-154, algebra/src/context.cpp:156-215):

* the query is trimmed to the stream's support; an empty result is the zero Lie
  (signature: the unit tensor);
* without an explicit resolution the query resolution is
  ``max(stream resolution, param_to_resolution(length) + 2)``;
* the query is dissected into maximal dyadic intervals at that resolution;
* a piece at the stream resolution is a cached leaf (the CBH of the events it
  contains); a coarser piece is the CBH of its two halves, recursively; a finer
  piece is replaced by the leaf it starts in when both start at the same point,
  and dropped otherwise;
* the pieces are combined by CBH (log of the product of their exponentials,
  then projected to the Hall basis); the signature is ``exp(l2t(log_signature))``.

B200 design.  The reference caches only the leaves and recomputes every coarser
piece by recursive CBH at query time.  Here the whole dyadic tree is built once
on the GPU: leaf signatures come from the batched signature kernel (level-1
increments) or from exp of the embedded Lie increments (general increments),
and every coarser node is the product of its children (one batched product
launch per level).  A query is then the ordered product of at most ~2 x
resolution cached node signatures (batched across queries, one launch per
piece position), followed by a float64 log and the Lie projection.  Since
``log``/``exp`` are mutually inverse on group-like elements and CBH is
associative, this equals the reference's CBH recursion up to rounding.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from . import compute as rpc
from . import signatures as S

__all__ = ["RealInterval", "DyadicInterval", "to_dyadic_intervals", "LieIncrementStream",
           "param_to_resolution"]


class RealInterval:
    """Half-open real interval; only clopen ``[inf, sup)`` is supported (as in RoughPy)."""

    def __init__(self, inf: float, sup: float, interval_type: str = "clopen"):
        if interval_type != "clopen":
            raise NotImplementedError("only clopen intervals are supported")
        self.inf = float(inf)
        self.sup = float(sup)
        self.type = interval_type

    def __repr__(self):
        return f"[{self.inf}, {self.sup})"


class DyadicInterval:
    """The clopen dyadic interval ``[k / 2^n, (k+1) / 2^n)``."""

    def __init__(self, k: int, n: int):
        self.k = int(k)
        self.n = int(n)

    @property
    def inf(self) -> float:
        return math.ldexp(self.k, -self.n)

    @property
    def sup(self) -> float:
        return math.ldexp(self.k + 1, -self.n)

    def __eq__(self, other):
        return isinstance(other, DyadicInterval) and (self.inf, self.sup) == (other.inf, other.sup)

    def __repr__(self):
        return f"DyadicInterval({self.k}, {self.n})"


def to_dyadic_intervals(interval: RealInterval, resolution: int) -> list:
    """Maximal dyadic dissection (intervals/src/dyadic_interval.cpp:191-224), via librpyb."""
    cap = 256
    k = np.zeros(cap, dtype=np.int64)
    p = np.zeros(cap, dtype=np.int32)
    n = int(_lib.lib.rpyb_dyadic_dissect(interval.inf, interval.sup, int(resolution), 1,
                                         k.ctypes.data, p.ctypes.data, cap))
    if n < 0:
        _lib.check(n)
    return [DyadicInterval(int(k[i]), int(p[i])) for i in range(n)]


def param_to_resolution(accuracy: float) -> int:
    """Resolution from the smallest index gap, as the Python bindings compute it
    (roughpy/src/args/kwargs_to_path_metadata.cpp:224-229)."""
    _, e = math.frexp(float(accuracy))
    return -min(5, e - 1)


def _query_param_to_resolution(length: float) -> int:
    """streams/include/roughpy/streams/stream_base.h:74-83"""
    _, e = math.frexp(float(length))
    return -min(0, e - 1)


def _dissect_batch(infs, sups, tols):
    n = len(infs)
    infs = np.ascontiguousarray(infs, dtype=np.float64)
    sups = np.ascontiguousarray(sups, dtype=np.float64)
    tols = np.ascontiguousarray(tols, dtype=np.int32)
    cap = int(max(1, n) * (2 * (int(tols.max()) if n else 0) + 130))
    k = np.zeros(cap, dtype=np.int64)
    p = np.zeros(cap, dtype=np.int32)
    off = np.zeros(n + 1, dtype=np.int64)
    _lib.check(_lib.lib.rpyb_dyadic_dissect_batch(n, infs.ctypes.data, sups.ctypes.data,
                                                  tols.ctypes.data, 1, k.ctypes.data,
                                                  p.ctypes.data, cap, off.ctypes.data))
    m = int(off[-1])
    return k[:m], p[:m], off


class LieIncrementStream:
    """Stream of Lie increments with a GPU-resident dyadic signature tree."""

    def __init__(self, times, lies, width, depth, resolution, support, dtype=np.float64,
                 mode=None, device="cuda"):
        self.width = int(width)
        self.depth = int(depth)
        self.resolution = int(resolution)
        self.support = support
        self.dtype = np.dtype(dtype)
        self.mode = mode or ("f64" if self.dtype == np.float64 else "f32c")
        self.device = torch.device(device)
        self.times = np.asarray(times, dtype=np.float64)
        self.lies = np.asarray(lies, dtype=np.float64)        # [n_events, lie_dim]
        self.tensor_basis = rpc.TensorBasis(self.width, self.depth)
        self.lie_basis = rpc.LieBasis(self.width, self.depth)
        self._tree = None

    # ------------------------------------------------------------- creation
    @classmethod
    def from_increments(cls, data, indices=None, width=None, depth=None, resolution=None,
                        dtype=None, support=None, mode=None, device="cuda", **kwargs):
        """Build a stream from increment rows (roughpy/src/streams/lie_increment_stream.cpp:73-246).

        ``data``: rows of Lie coordinates (the first ``width`` are the letters;
        further entries are higher Hall-basis coordinates) or a sequence of
        arrays.  ``indices``: event times (default 0, 1, 2, ... with
        resolution 0).  Without an explicit resolution the reference's
        heuristic is reproduced, including its use of the smallest index
        rather than the smallest gap.
        """
        coeffs = kwargs.pop("coeffs", None)
        if kwargs:
            raise TypeError(f"unexpected keyword arguments {sorted(kwargs)}")
        if dtype is None and coeffs is not None:
            dtype = {"DPReal": np.float64, "SPReal": np.float32}.get(str(coeffs), None)
        rows = np.asarray(data)
        if rows.ndim == 1:
            rows = rows.reshape(1, -1)
        if rows.ndim != 2:
            raise ValueError("increments must be a two-dimensional array")
        if dtype is None:
            dtype = np.float32 if rows.dtype == np.float32 else np.float64
        if width is None:
            width = rows.shape[1]
        if not width or not depth:
            raise ValueError("either ctx or both width and depth must be specified")
        lie_dim = rpc.LieBasis(width, depth).size()
        lies = np.zeros((rows.shape[0], lie_dim), dtype=np.float64)
        ncol = min(rows.shape[1], lie_dim)
        lies[:, :ncol] = rows[:, :ncol]
        n = rows.shape[0]
        if indices is None:
            idx = np.arange(n, dtype=np.float64)
            res = 0 if resolution is None else int(resolution)
        else:
            idx = np.asarray(indices, dtype=np.float64).reshape(-1)
            if idx.shape[0] != n:
                raise ValueError("mismatch between number of rows in data and number of indices")
            if resolution is None:
                # lie_increment_stream.cpp:193-205 (the gap is measured from 0)
                min_diff = math.inf
                res = 0
                for v in idx:
                    min_diff = min(min_diff, v - 0.0)
                    res = param_to_resolution(min_diff) + 1
            else:
                res = int(resolution)
        # first event wins at duplicate times (flat_map::try_emplace)
        order = np.argsort(idx, kind="stable")
        t_sorted = idx[order]
        keep = np.ones(n, dtype=bool)
        keep[1:] = t_sorted[1:] != t_sorted[:-1]
        times = t_sorted[keep]
        lies = lies[order][keep]
        if support is None:
            if n:
                support = RealInterval(float(idx.min()), float(idx.max()) + math.ldexp(1.0, -res))
            else:
                support = RealInterval(0.0, 1.0)
        elif not isinstance(support, RealInterval):
            support = RealInterval(*support)
        return cls(times, lies, width, depth, res, support, dtype, mode, device)

    # ------------------------------------------------------------- the tree
    @property
    def _sig_dtype(self):
        return torch.float64 if self.mode == "f64" else torch.float32

    def _build_tree(self):
        """All dyadic nodes at and above the stream resolution, on the GPU.

        Level j holds the aligned blocks of 2^j leaves intersecting the leaf
        range [m_lo, m_hi]: block b covers leaves [b 2^j, (b+1) 2^j), which is
        the dyadic interval (b, resolution - j).  Block ranges follow floor
        division, so supports on both sides of 0 (where no dyadic interval
        spans the origin) work too.  The last row of the tree is the unit,
        standing in for children outside the range.
        """
        if self._tree is not None:
            return self._tree
        R = self.resolution
        s0, s1 = self.support.inf, self.support.sup
        m_lo = math.floor(math.ldexp(s0, R))
        m_hi = max(m_lo, math.ceil(math.ldexp(s1, R)) - 1)
        if self.times.size:
            m_lo = min(m_lo, math.floor(math.ldexp(float(self.times.min()), R)))
            m_hi = max(m_hi, math.floor(math.ldexp(float(self.times.max()), R)))
        lo, cnt, base = [], [], []
        rows = 0
        j = 0
        while True:
            l_j, h_j = m_lo >> j, m_hi >> j
            # a range on both sides of 0 stops merging at blocks -1 and 0
            if j > 0 and l_j == -1 and h_j == 0 and cnt[-1] == 2:
                break
            lo.append(l_j)
            cnt.append(h_j - l_j + 1)
            base.append(rows)
            rows += h_j - l_j + 1
            if h_j == l_j:
                break
            j += 1
            if j > 62:
                raise ValueError("stream support too wide for its resolution")
        J = len(lo) - 1
        unit_row = rows
        rows += 1
        T = self.tensor_basis.size()
        dt = self._sig_dtype
        dev = self.device
        code = _lib.F64 if dt == torch.float64 else _lib.F32
        tree = torch.empty((rows, T), dtype=dt, device=dev)
        tree[unit_row].zero_()
        tree[unit_row, 0] = 1.0
        # leaves: events grouped by leaf, Chen product of exp(increment)
        n_leaves = cnt[0]
        leaf_of = np.floor(np.ldexp(self.times, R)).astype(np.int64) - m_lo
        off = np.searchsorted(leaf_of, np.arange(n_leaves + 1), side="left").astype(np.int64)
        leaves = tree[:n_leaves]
        higher = self.lies[:, self.width:]
        if higher.size == 0 or not np.any(higher):
            inc = torch.from_numpy(np.ascontiguousarray(self.lies[:, :self.width])).to(dev, dt)
            plan = S.SignaturePlan(off, self.width, self.depth, self.mode, device=dev)
            plan.run(inc.contiguous(), leaves)
        else:
            self._general_leaves(leaves, off, code)
        # level j node b = child (j-1, 2b) * child (j-1, 2b+1)
        stream = torch.cuda.current_stream(dev).cuda_stream
        for j in range(1, J + 1):
            b = np.arange(lo[j], lo[j] + cnt[j], dtype=np.int64)
            kids = []
            for c in (2 * b, 2 * b + 1):
                inside = (c >= lo[j - 1]) & (c < lo[j - 1] + cnt[j - 1])
                kids.append(np.where(inside, base[j - 1] + (c - lo[j - 1]), unit_row))
            out_idx = torch.from_numpy(base[j] + (b - lo[j])).to(dev)
            lhs_idx = torch.from_numpy(kids[0]).to(dev)
            rhs_idx = torch.from_numpy(kids[1]).to(dev)
            _lib.check(_lib.lib.rpyb_ft_mul_gather(
                code, self.width, self.depth, cnt[j], tree.data_ptr(), tree.data_ptr(),
                tree.data_ptr(), T, out_idx.data_ptr(), lhs_idx.data_ptr(),
                rhs_idx.data_ptr(), 0, stream))
        self._tree = dict(tensor=tree, J=J, lo=lo, cnt=cnt, base=base, unit_row=unit_row)
        return self._tree

    def _general_leaves(self, leaves, off, code):
        """Leaves for increments with higher Hall coordinates: Π exp(l2t(lie))."""
        dev = self.device
        dt = leaves.dtype
        T = self.tensor_basis.size()
        l2t = self.lie_basis.get_l2t_matrix()
        lies = torch.from_numpy(np.ascontiguousarray(self.lies)).to(dev, dt)
        emb = torch.zeros((lies.shape[0], T), dtype=dt, device=dev)
        if lies.shape[0]:
            rpc._internals.dense_lie_to_tensor(emb, lies, l2t, self.lie_basis, self.tensor_basis)
        ex = torch.zeros_like(emb)
        if lies.shape[0]:
            rpc._internals.dense_ft_exp(ex, emb, self.tensor_basis)
        counts = np.diff(off)
        leaves.zero_()
        leaves[:, 0] = 1.0
        _ordered_products(leaves, ex, off, counts, code, self.width, self.depth)

    # ------------------------------------------------------------- queries
    def _pieces(self, infs, sups, resolution):
        """Per query: node rows of the tree, in order (zero pieces dropped)."""
        tr = self._build_tree()
        R, J = self.resolution, tr["J"]
        s0, s1 = self.support.inf, self.support.sup
        n = len(infs)
        qi = np.empty(n)
        qs = np.empty(n)
        tols = np.empty(n, dtype=np.int32)
        empty = np.zeros(n, dtype=bool)
        for q in range(n):
            a, b = float(infs[q]), float(sups[q])
            if a > b:
                raise ValueError("inf must not be larger than sup")
            # stream.cpp:37-52 check_support_and_trim, :54-71 refine_interval
            if b < s0 or a > s1:
                empty[q] = True
                a = b = s0
            else:
                a, b = max(a, s0), min(b, s1)
            if b - a == 0.0:
                empty[q] = True
            qi[q], qs[q] = a, b
            if resolution is None:
                tols[q] = max(R, _query_param_to_resolution(b - a) + 2) if not empty[q] else R
            else:
                tols[q] = int(resolution)
        k, p, off = _dissect_batch(qi, qs, tols)
        nodes = np.full(k.shape[0], -1, dtype=np.int64)
        lo = np.asarray(tr["lo"], dtype=np.int64)
        cnt = np.asarray(tr["cnt"], dtype=np.int64)
        base = np.asarray(tr["base"], dtype=np.int64)

        def node_rows(level, blk):
            ok = (level >= 0) & (level <= J)
            lv = np.clip(level, 0, J)
            rel = blk - lo[lv]
            ok &= (rel >= 0) & (rel < cnt[lv])
            return np.where(ok, base[lv] + rel, -1)

        # dyadic_caching_layer.cpp:86-130: at the stream resolution a cached leaf;
        # coarser pieces are whole tree nodes (the CBH of their halves); a finer
        # piece maps to the leaf it starts in when the start points coincide
        # (rational_equals on the included ends) and is dropped otherwise.
        at = p <= R
        nodes[at] = node_rows((R - p[at]).astype(np.int64), k[at])
        fine = p > R
        if np.any(fine):
            sh = (p[fine] - R).astype(np.int64)
            kk = k[fine]
            tk = kk >> sh
            same = (tk << sh) == kk
            nodes[fine] = np.where(same, node_rows(np.zeros_like(tk), tk), -1)
        for q in np.nonzero(empty)[0]:
            nodes[off[q]:off[q + 1]] = -1
        return nodes, off

    def _query_products(self, infs, sups, resolution):
        tr = self._build_tree()
        tree = tr["tensor"]
        nodes, off = self._pieces(infs, sups, resolution)
        n = len(infs)
        # drop zero pieces, keep order
        keep = nodes >= 0
        cs = np.zeros(nodes.shape[0] + 1, dtype=np.int64)
        np.cumsum(keep, out=cs[1:])
        counts = cs[off[1:]] - cs[off[:-1]]
        kept = nodes[keep]
        koff = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(counts, out=koff[1:])
        T = self.tensor_basis.size()
        # queries accumulate in float64; float32 nodes enter through the mixed product
        acc = torch.zeros((n, T), dtype=torch.float64, device=self.device)
        acc[:, 0] = 1.0
        _ordered_products(acc, tree, koff, counts, None, self.width, self.depth, src_rows=kept)
        return acc

    def _log_signature_batch(self, infs, sups, resolution=None):
        prods = self._query_products(infs, sups, resolution)
        p64 = prods
        logs = torch.zeros_like(p64)
        rpc._internals.dense_ft_log(logs, p64, self.tensor_basis)
        lie = torch.zeros((p64.shape[0], self.lie_basis.size()), dtype=torch.float64,
                          device=self.device)
        rpc._internals.dense_tensor_to_lie(lie, logs, self.lie_basis.get_t2l_matrix(),
                                           self.lie_basis, self.tensor_basis)
        return lie

    def log_signature_batch(self, infs, sups, resolution=None, chunk=16384):
        """Log-signatures (Hall coordinates, float64) of many clopen intervals."""
        infs = np.asarray(infs, dtype=np.float64).reshape(-1)
        sups = np.asarray(sups, dtype=np.float64).reshape(-1)
        outs = [self._log_signature_batch(infs[i:i + chunk], sups[i:i + chunk], resolution)
                for i in range(0, infs.shape[0], chunk)]
        if not outs:
            return torch.zeros((0, self.lie_basis.size()), dtype=torch.float64, device=self.device)
        return torch.cat(outs)

    def signature_batch(self, infs, sups, resolution=None, chunk=16384):
        """Signatures exp(l2t(log_signature)) (float64) of many clopen intervals."""
        lie = self.log_signature_batch(infs, sups, resolution, chunk)
        return self._to_signature(lie)

    def _to_signature(self, lie):
        # algebra/src/context.cpp:156-159: exp(lie_to_tensor(log_signature))
        T = self.tensor_basis.size()
        emb = torch.zeros((lie.shape[0], T), dtype=torch.float64, device=self.device)
        rpc._internals.dense_lie_to_tensor(emb, lie, self.lie_basis.get_l2t_matrix(),
                                           self.lie_basis, self.tensor_basis)
        sig = torch.zeros_like(emb)
        rpc._internals.dense_ft_exp(sig, emb, self.tensor_basis)
        return sig

    def _interval_args(self, interval_or_inf, sup):
        if interval_or_inf is None:
            return self.support.inf, self.support.sup
        if isinstance(interval_or_inf, (RealInterval, DyadicInterval)):
            return interval_or_inf.inf, interval_or_inf.sup
        if sup is None:
            raise TypeError("expected an interval or an inf, sup pair")
        if float(interval_or_inf) > float(sup):
            raise ValueError("inf must not be larger than sup")
        return float(interval_or_inf), float(sup)

    def _truncate_lie(self, lie, depth):
        if depth is None or depth >= self.depth:
            return lie
        return lie[..., :int(self.lie_basis.degree_begin[depth + 1]) - 1]

    def _truncate_tensor(self, t, depth):
        if depth is None or depth >= self.depth:
            return t
        return t[..., :int(self.tensor_basis.degree_begin[depth + 1])]

    def log_signature(self, interval_or_inf=None, sup=None, resolution=None, depth=None):
        """Log-signature over an interval (streams/src/stream.cpp:125-154), float64 numpy."""
        a, b = self._interval_args(interval_or_inf, sup)
        lie = self._log_signature_batch(np.array([a]), np.array([b]), resolution)
        return self._truncate_lie(lie[0].cpu().numpy(), depth)

    def signature(self, interval_or_inf=None, sup=None, resolution=None, depth=None):
        """Signature over an interval (streams/src/stream.cpp:156-171), float64 numpy."""
        a, b = self._interval_args(interval_or_inf, sup)
        lie = self._log_signature_batch(np.array([a]), np.array([b]), resolution)
        return self._truncate_tensor(self._to_signature(lie)[0].cpu().numpy(), depth)


def _ordered_products(acc, src, off, counts, code, width, depth, src_rows=None):
    """acc[q] <- acc[q] * src[r_0] * src[r_1] * ... over q's rows (in order).

    Rows of q are src_rows[off[q]:off[q+1]] (or the range itself when
    src_rows is None).  One batched product launch per position.
    """
    n = acc.shape[0]
    if n == 0:
        return
    dev = acc.device
    T = acc.shape[1]
    counts = np.asarray(counts, dtype=np.int64)
    maxc = int(counts.max()) if counts.size else 0
    if src_rows is None:
        src_rows = np.arange(int(off[-1]), dtype=np.int64)
    mixed = acc.dtype == torch.float64 and src.dtype == torch.float32
    if not mixed and acc.dtype != src.dtype:
        raise TypeError("unsupported dtype combination")
    if code is None:
        code = _lib.F64 if acc.dtype == torch.float64 else _lib.F32
    tmp = torch.empty_like(acc)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for r in range(maxc):
        active = np.nonzero(counts > r)[0]
        m = active.shape[0]
        rows = src_rows[off[active] + r]
        q_t = torch.from_numpy(active.astype(np.int64)).to(dev)
        out_t = torch.arange(m, device=dev, dtype=torch.int64)
        r_t = torch.from_numpy(rows).to(dev)
        if mixed:
            rc = _lib.lib.rpyb_ft_mul_gather_mixed(width, depth, m, tmp.data_ptr(), acc.data_ptr(),
                                                   src.data_ptr(), T, out_t.data_ptr(),
                                                   q_t.data_ptr(), r_t.data_ptr(), 0, stream)
        else:
            rc = _lib.lib.rpyb_ft_mul_gather(code, width, depth, m, tmp.data_ptr(),
                                             acc.data_ptr(), src.data_ptr(), T, out_t.data_ptr(),
                                             q_t.data_ptr(), r_t.data_ptr(), 0, stream)
        _lib.check(rc)
        acc.index_copy_(0, q_t, tmp[:m])
