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
on the GPU by the native runtime behind the C ABI (``rpyb_dyadic_build``): leaf
signatures come from the batched signature kernel (level-1 increments) or from
exp of the embedded Lie increments (general increments), and every coarser node
is the product of its children (one batched product launch per level).  A query
batch (``rpyb_dyadic_query``) is trimmed and dissected on the host, then each
query is the ordered product of at most ~2 x resolution cached node signatures
(batched across queries, one launch per piece position), followed by a float64
log and the Lie projection.  Since ``log``/``exp`` are mutually inverse on
group-like elements and CBH is associative, this equals the reference's CBH
recursion up to rounding.  This module keeps the reference's construction
rules (event de-duplication, the resolution heuristic, the default support).
"""
from __future__ import annotations

import copy
import ctypes
import json
import math

import numpy as np
import torch

from . import _lib
from . import compute as rpc
from . import signatures as S

__all__ = ["RealInterval", "DyadicInterval", "Partition", "to_dyadic_intervals",
           "LieIncrementStream", "TickStream", "PiecewiseAbelianStream", "param_to_resolution",
           "sig_derivative", "sig_derivative_batch"]


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


class Partition:
    """A clopen interval cut at intermediate points (intervals/src/partition.cpp:
    the points strictly inside the interval are kept, sorted, duplicates
    included); ``partition[i]`` is the i-th sub-interval."""

    def __init__(self, interval, intermediates=()):
        inf, sup = ((interval.inf, interval.sup) if isinstance(interval, (RealInterval,))
                    else (float(interval[0]), float(interval[1])))
        self.inf, self.sup = float(inf), float(sup)
        self._points = sorted(float(m) for m in intermediates
                              if self.inf <= float(m) < self.sup and float(m) != self.inf)

    def __len__(self):
        return len(self._points) + 1

    def __getitem__(self, i):
        n = len(self._points)
        if i < 0:
            i += n + 1
        if not 0 <= i <= n:
            raise IndexError("partition index out of range")
        lo = self.inf if i == 0 else self._points[i - 1]
        hi = self.sup if i == n else self._points[i]
        return RealInterval(lo, hi)

    def intermediates(self):
        return list(self._points)

    def __eq__(self, other):
        return (isinstance(other, Partition) and (self.inf, self.sup) == (other.inf, other.sup)
                and self._points == other._points)

    def __repr__(self):
        ends = [self.inf] + self._points + [self.sup]
        return "{" + ", ".join(f"[{a}, {b})" for a, b in zip(ends[:-1], ends[1:])) + "}"

    def mesh(self):
        """Length of the largest sub-interval."""
        ends = [self.inf] + self._points + [self.sup]
        return max(b - a for a, b in zip(ends[:-1], ends[1:]))

    def refine_midpoints(self):
        """The partition with the midpoint of every sub-interval added."""
        ends = [self.inf] + self._points + [self.sup]
        mids = [(a + b) / 2.0 for a, b in zip(ends[:-1], ends[1:])]
        return Partition(RealInterval(self.inf, self.sup), self._points + mids)


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


def _resolution_arg(resolution):
    """A query's resolution argument as the bindings read it
    (roughpy/src/streams/signature_arguments.cpp:30-50): None keeps the
    default, an int is the resolution, a float is an accuracy turned into a
    resolution by param_to_resolution."""
    if resolution is None:
        return None
    if isinstance(resolution, (bool, np.bool_)):
        raise TypeError("resolution should be either float or int")
    if isinstance(resolution, (int, np.integer)):
        return int(resolution)
    if isinstance(resolution, (float, np.floating)):
        return param_to_resolution(float(resolution))
    raise TypeError("resolution should be either float or int")


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


class _StreamQueries:
    """Query front end shared by the stream classes (the reference's
    Stream::log_signature / signature / signature_derivative and its Python
    argument rules, roughpy/src/streams/signature_arguments.cpp:56-160).
    Subclasses provide ``_query(infs, sups, resolution, logsig, sig)``."""

    def _interval_args(self, interval_or_inf, sup, resolution=None):
        """(inf, sup, resolution): an interval, an inf/sup pair, nothing (the
        whole support) or an integer alone (a resolution over the support).
        After an interval the second argument is the resolution; a float
        resolution is an accuracy (signature_arguments.cpp:30-50, :95-170)."""
        if interval_or_inf is None:
            return self.support.inf, self.support.sup, _resolution_arg(resolution)
        if isinstance(interval_or_inf, (RealInterval, DyadicInterval)):
            if sup is not None:
                resolution = sup
            return interval_or_inf.inf, interval_or_inf.sup, _resolution_arg(resolution)
        if sup is None:
            if isinstance(interval_or_inf, (int, np.integer)) and not isinstance(interval_or_inf, bool):
                return self.support.inf, self.support.sup, int(interval_or_inf)
            raise TypeError("expecting integer resolution")
        if not isinstance(sup, (int, float, np.integer, np.floating)) or isinstance(sup, bool):
            raise TypeError("expected float value for sup")
        if float(interval_or_inf) > float(sup):
            raise ValueError("inf must not be larger than sup")
        return float(interval_or_inf), float(sup), _resolution_arg(resolution)

    def _truncate_lie(self, lie, depth):
        if depth is None or depth >= self.depth:
            return lie
        return lie[..., :int(self.lie_basis.degree_begin[depth + 1]) - 1]

    def _truncate_tensor(self, t, depth):
        if depth is None or depth >= self.depth:
            return t
        return t[..., :int(self.tensor_basis.degree_begin[depth + 1])]

    def log_signature_batch(self, infs, sups, resolution=None, chunk=16384):
        """Log-signatures (Hall coordinates, float64) of many clopen intervals."""
        resolution = _resolution_arg(resolution)
        infs = np.asarray(infs, dtype=np.float64).reshape(-1)
        sups = np.asarray(sups, dtype=np.float64).reshape(-1)
        outs = [self._query(infs[i:i + chunk], sups[i:i + chunk], resolution)[0]
                for i in range(0, infs.shape[0], chunk)]
        if not outs:
            return torch.zeros((0, self.lie_basis.size()), dtype=torch.float64, device=self.device)
        return torch.cat(outs)

    def signature_batch(self, infs, sups, resolution=None, chunk=16384):
        """Signatures exp(l2t(log_signature)) (float64) of many clopen intervals."""
        resolution = _resolution_arg(resolution)
        infs = np.asarray(infs, dtype=np.float64).reshape(-1)
        sups = np.asarray(sups, dtype=np.float64).reshape(-1)
        outs = [self._query(infs[i:i + chunk], sups[i:i + chunk], resolution, False, True)[1]
                for i in range(0, infs.shape[0], chunk)]
        if not outs:
            return torch.zeros((0, self.tensor_basis.size()), dtype=torch.float64,
                               device=self.device)
        return torch.cat(outs)

    def _log_signature_batch(self, infs, sups, resolution=None):
        return self._query(infs, sups, resolution)[0]

    def log_signature(self, interval_or_inf=None, sup=None, resolution=None, depth=None):
        """Log-signature over an interval (streams/src/stream.cpp:125-154), float64 numpy."""
        a, b, res = self._interval_args(interval_or_inf, sup, resolution)
        lie = self._query(np.array([a]), np.array([b]), res)[0]
        return self._truncate_lie(lie[0].cpu().numpy(), depth)

    def signature(self, interval_or_inf=None, sup=None, resolution=None, depth=None):
        """Signature over an interval (streams/src/stream.cpp:156-171), float64 numpy."""
        a, b, res = self._interval_args(interval_or_inf, sup, resolution)
        sig = self._query(np.array([a]), np.array([b]), res, False, True)[1]
        return self._truncate_tensor(sig[0].cpu().numpy(), depth)

    def restrict(self, interval):
        """The same stream with its support replaced by ``interval``
        (streams/src/stream.cpp:73-89, Stream::restrict): later queries are
        trimmed to the new support, not to its intersection with the old
        one.  The events are shared; a device tree is built again for the
        new support on first use, since queries are trimmed where the tree
        was built."""
        inf, sup = ((interval.inf, interval.sup)
                    if isinstance(interval, (RealInterval, DyadicInterval)) else interval)
        new = copy.copy(self)
        new._base_support = getattr(self, "_base_support", self.support)
        new.support = RealInterval(float(inf), float(sup))
        if hasattr(new, "_tree"):
            new._tree = None
        return new

    def simplify(self, partition, resolution=None, ctx=None, depth=None):
        """A PiecewiseAbelianStream with one piece per interval of
        ``partition``: the interval's log-signature at ``resolution``
        (default: the stream's) (streams/src/stream.cpp:232-258).  As in the
        reference the new stream keeps the underlying stream's own support
        (not one set by ``restrict``) and takes ``resolution`` as its
        default; ``ctx.depth`` (a context wins over ``depth``, and its width
        must be the stream's) or ``depth`` truncates the pieces.  A depth
        above the stream's is rejected: the device tree holds the stream's
        depth only, where the reference would build a deeper context."""
        if not isinstance(partition, Partition):
            partition = Partition(*partition)
        # the binding parses resolution and depth as C ints ("i"): a float is
        # a TypeError there, and a context takes precedence over depth
        for name, v in (("resolution", resolution), ("depth", depth)):
            if v is not None and not isinstance(v, (int, np.integer)):
                raise TypeError(f"{name} must be an integer, not {type(v).__name__}")
        if ctx is not None:
            if int(getattr(ctx, "width", self.width)) != self.width:
                raise ValueError("context width must match stream width")
            depth = getattr(ctx, "depth", None)
        res = self.resolution if resolution is None else int(resolution)
        if depth and int(depth) > self.depth:
            # the reference would build a deeper context (get_alike); the
            # device tree holds the stream's depth only
            raise ValueError(f"depth {int(depth)} exceeds the stream's depth {self.depth}")
        d = self.depth if not depth else int(depth)
        ivs = [partition[i] for i in range(len(partition))]
        infs = np.array([iv.inf for iv in ivs])
        sups = np.array([iv.sup for iv in ivs])
        lies = self._query(infs, sups, res)[0].cpu().numpy()
        lies = lies[:, :rpc.LieBasis(self.width, d).size()]
        support = getattr(self, "_base_support", self.support)
        return PiecewiseAbelianStream(infs, sups, lies, self.width, d, res,
                                      RealInterval(support.inf, support.sup), self.device)

    def signature_derivative(self, interval, perturbation=None, resolution=None, depth=None):
        """Derivative of the signature along Lie perturbations
        (streams/src/stream.cpp:173-230): ``interval`` with one
        ``perturbation`` (Hall coordinates), or a list of (interval,
        perturbation) pairs.  Each interval's log-signature comes from the
        stream's queries; float64 numpy tensor."""
        resolution = _resolution_arg(resolution)
        pairs = list(interval) if perturbation is None else [(interval, perturbation)]
        ivs = [self._interval_args(iv, None) if isinstance(iv, (RealInterval, DyadicInterval))
               else self._interval_args(*iv) for iv, _ in pairs]
        a = np.array([v[0] for v in ivs])
        b = np.array([v[1] for v in ivs])
        lies = self._query(a, b, resolution)[0]
        L = self.lie_basis.size()
        pert = np.zeros((len(pairs), L))
        for i, (_, p) in enumerate(pairs):
            p = np.asarray(getattr(p, "data", p), dtype=np.float64).reshape(-1)
            pert[i, :min(L, p.size)] = p[:L]
        out = sig_derivative_batch(lies, pert, [0, len(pairs)], self.width, self.depth,
                                   self.device)
        return self._truncate_tensor(out[0].cpu().numpy(), depth)


class LieIncrementStream(_StreamQueries):
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
        # [n_events, c] Hall coordinates of the events, c <= lie_dim (omitted
        # trailing coordinates are zero)
        self.lies = np.asarray(lies, dtype=np.float64)
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
        ncol = min(rows.shape[1], lie_dim)
        lies = np.zeros((rows.shape[0], max(ncol, width)), dtype=np.float64)
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
        """The device dyadic tree (``rpyb_dyadic_build``), built on first use."""
        if self._tree is not None:
            return self._tree
        dt = self._sig_dtype
        code = _lib.F64 if dt == torch.float64 else _lib.F32
        higher = self.lies[:, self.width:]
        if higher.size == 0 or not np.any(higher):
            rows, row_len = self.lies[:, :self.width], self.width
        else:
            L = self.lie_basis.size()
            rows = np.zeros((self.lies.shape[0], L))
            rows[:, :self.lies.shape[1]] = self.lies
            row_len = L
        n = int(self.times.shape[0])
        rows_t = torch.from_numpy(np.ascontiguousarray(rows)).to(self.device, dt).contiguous()
        times = np.ascontiguousarray(self.times, dtype=np.float64)
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _lib.check(_lib.lib.rpyb_dyadic_build(
                code, self.width, self.depth, self.resolution, float(self.support.inf),
                float(self.support.sup), n, times.ctypes.data if n else None,
                rows_t.data_ptr() if n else None, row_len, ctypes.byref(handle), stream))
        self._tree = _DyadicTree(handle, self.device)
        return self._tree

    def build_range_table(self, block_log2: int = 0) -> None:
        """Build the tree's range-product table (``rpyb_dyadic_range_table``):
        queries spanning more than one block of leaves then multiply at most
        four table rows instead of every dyadic piece.  Done automatically at
        the first batch of 1024 or more queries on a tree of 4096 or more
        leaves (``auto_range_table``)."""
        tr = self._build_tree()
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _lib.check(_lib.lib.rpyb_dyadic_range_table(tr.handle, int(block_log2), stream))
        tr.refresh()
        tr.range_table = True

    auto_range_table = True

    # ------------------------------------------------------------- persistence
    def save(self, path) -> None:
        """Write the stream (events, shape, resolution, support) and its
        device dyadic tree (``rpyb_dyadic_save``) to ``path`` (an ``.npz``
        archive).  The analogue of the reference's cache dump
        (streams/src/dyadic_caching_layer.cpp:168-201)."""
        tr = self._build_tree()
        size = int(_lib.lib.rpyb_dyadic_save_size(tr.handle))
        if size < 0:
            _lib.check(size)
        blob = np.empty(size, dtype=np.uint8)
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            got = int(_lib.lib.rpyb_dyadic_save(tr.handle, blob.ctypes.data, size, stream))
        if got < 0:
            _lib.check(got)
        meta = {"kind": type(self).__name__, "width": self.width, "depth": self.depth,
                "resolution": self.resolution, "support": [self.support.inf, self.support.sup],
                "dtype": self.dtype.name, "mode": self.mode}
        np.savez(path, meta=np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8),
                 times=self.times, lies=self.lies, tree=blob)

    @classmethod
    def load(cls, path, device="cuda"):
        """A stream written by ``save``; its tree is loaded onto ``device``
        (``rpyb_dyadic_load``) instead of being rebuilt."""
        with np.load(path) as z:
            meta = json.loads(bytes(z["meta"]).decode())
            times, lies, blob = z["times"], z["lies"], np.ascontiguousarray(z["tree"])
        if meta.get("kind") != cls.__name__:
            raise TypeError(f"{path} holds a {meta.get('kind')}, not a {cls.__name__}")
        st = cls(times, lies, meta["width"], meta["depth"], meta["resolution"],
                 RealInterval(*meta["support"]), np.dtype(meta["dtype"]), meta["mode"], device)
        handle = ctypes.c_void_p()
        with torch.cuda.device(st.device):
            stream = torch.cuda.current_stream(st.device).cuda_stream
            _lib.check(_lib.lib.rpyb_dyadic_load(blob.ctypes.data, blob.size,
                                                 ctypes.byref(handle), stream))
        st._tree = _DyadicTree(handle, st.device)
        return st

    # ------------------------------------------------------------- queries
    def _query(self, infs, sups, resolution, logsig=True, sig=False):
        """One rpyb_dyadic_query over clopen intervals; float64 device outputs."""
        tr = self._build_tree()
        infs = np.ascontiguousarray(infs, dtype=np.float64).reshape(-1)
        if (self.auto_range_table and not tr.range_table and infs.shape[0] >= 1024
                and tr.rows >= 8192):
            self.build_range_table()
        sups = np.ascontiguousarray(sups, dtype=np.float64).reshape(-1)
        n = infs.shape[0]
        L, T = self.lie_basis.size(), self.tensor_basis.size()
        lie = torch.empty((n, L), dtype=torch.float64, device=self.device) if logsig else None
        sg = torch.empty((n, T), dtype=torch.float64, device=self.device) if sig else None
        if n == 0:
            return lie, sg
        res = _lib.QUERY_RESOLUTION_AUTO if resolution is None else int(resolution)
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _lib.check(_lib.lib.rpyb_dyadic_query(
                tr.handle, n, infs.ctypes.data, sups.ctypes.data, res,
                lie.data_ptr() if logsig else None, L, sg.data_ptr() if sig else None, T,
                stream))
        return lie, sg


class TickStream(LieIncrementStream):
    """Tick stream (streams/src/tick_stream.cpp:41-201,
    streams/include/roughpy/streams/tick_stream.h:66-83): events (time, Lie
    coordinates) keyed by their dyadic interval at the stream resolution.
    Events sharing an interval are combined in input order and are not
    de-duplicated by time; a dyadic query piece takes the log-signature of
    the events inside it (the reference looks up the cached CBH of the
    smallest dyadic interval holding them), and the pieces are combined as
    for every stream (streams/src/stream.cpp:37-171).

    On the device this is the dyadic signature tree of the events sorted
    stably by interval, each placed at its interval's start: a leaf is the
    product of exp over its events in input order, every node the product of
    the events inside it, so the queries are those of LieIncrementStream.
    The reference's construction does not terminate when there are events
    both before 0 and in the interval starting at 0 (its search for the
    smallest interval holding the negative events cannot pass 0); that case
    has a well-defined answer here."""

    @classmethod
    def from_lie_events(cls, times, data, width, depth, resolution=0, support=None, dtype=None,
                        mode=None, device="cuda"):
        """The stream of events (times[i], data[i]), in input order.

        ``data``: rows of Lie coordinates (the first ``width`` are the letters;
        further entries are higher Hall-basis coordinates).  ``resolution``
        and ``support`` default as in the reference's tick-stream
        constructor: 0 and [0, 1) (roughpy/src/streams/tick_stream.cpp:131-141).
        """
        rows = np.asarray(data)
        if rows.ndim == 1:
            rows = rows.reshape(1, -1)
        if rows.ndim != 2:
            raise ValueError("tick data must be a two-dimensional array")
        t = np.asarray(times, dtype=np.float64).reshape(-1)
        if t.shape[0] != rows.shape[0]:
            raise ValueError("mismatch between number of rows in data and number of times")
        if t.shape[0] == 0:
            raise ValueError("tick data cannot be empty")
        if dtype is None:
            dtype = np.float32 if rows.dtype == np.float32 else np.float64
        lie_dim = rpc.LieBasis(width, depth).size()
        ncol = min(rows.shape[1], lie_dim)
        lies = np.zeros((rows.shape[0], max(ncol, width)), dtype=np.float64)
        lies[:, :ncol] = rows[:, :ncol]
        res = int(resolution)
        # DyadicInterval(t, resolution): [floor(t 2^res), +1) / 2^res
        k = np.floor(np.ldexp(t, res))
        order = np.argsort(k, kind="stable")
        starts = np.ldexp(k[order], -res)
        if support is None:
            support = RealInterval(0.0, 1.0)
        elif not isinstance(support, RealInterval):
            support = RealInterval(*support)
        return cls(starts, lies[order], width, depth, res, support, dtype, mode, device)

    @classmethod
    def from_increments(cls, *args, **kwargs):
        # LieIncrementStream's constructor de-duplicates event times, which a
        # tick stream does not
        raise TypeError("a TickStream is built with TickStream.from_lie_events")

    @classmethod
    def from_data(cls, *args, **kwargs):
        raise NotImplementedError(
            "tick data parsing (labels, channel types, schemas) is not provided; build the "
            "stream from (time, Lie coordinates) events with TickStream.from_lie_events")


class PiecewiseAbelianStream(_StreamQueries):
    """A stream given as (interval, Lie element) pieces: RoughPy's
    PiecewiseAbelianStream (streams/src/piecewise_abelian_stream.cpp), built
    by ``construct`` as roughpy/src/streams/piecewise_abelian_stream.cpp:51-95
    does (support = hull of the pieces, resolution 0 unless given).  Queries
    run through ``rpyb_piecewise_query``."""

    def __init__(self, infs, sups, lies, width, depth, resolution, support, device="cuda"):
        self.width, self.depth = int(width), int(depth)
        self.resolution = int(resolution)
        self.support = support
        self.device = torch.device(device)
        self.tensor_basis = rpc.TensorBasis(self.width, self.depth)
        self.lie_basis = rpc.LieBasis(self.width, self.depth)
        self.piece_inf = np.ascontiguousarray(infs, dtype=np.float64)
        self.piece_sup = np.ascontiguousarray(sups, dtype=np.float64)
        self.pieces = torch.from_numpy(np.ascontiguousarray(lies, dtype=np.float64)).to(self.device)

    @classmethod
    def construct(cls, data, width=None, depth=None, resolution=None, dtype=None, ctx=None,
                  device="cuda", **kwargs):
        """``data``: (interval, Lie) pairs, the interval a RealInterval or an
        (inf, sup) pair, the Lie element its Hall coordinates."""
        if ctx is not None:
            width = width or getattr(ctx, "width", None)
            depth = depth or getattr(ctx, "depth", None)
        if kwargs:
            raise TypeError(f"unexpected keyword arguments {sorted(kwargs)}")
        if not width or not depth:
            raise ValueError("cannot deduce width/depth/ctype")
        L = rpc.LieBasis(width, depth).size()
        infs, sups, lies = [], [], []
        for iv, lie in data:
            a, b = (iv.inf, iv.sup) if isinstance(iv, (RealInterval, DyadicInterval)) else iv
            infs.append(float(a))
            sups.append(float(b))
            v = np.asarray(getattr(lie, "data", lie), dtype=np.float64).reshape(-1)
            row = np.zeros(L)
            row[:min(L, v.size)] = v[:L]
            lies.append(row)
        if infs:
            support = RealInterval(min(infs), max(sups))
        else:
            support = RealInterval(0.0, 1.0)
        lies = np.stack(lies) if lies else np.zeros((0, L))
        return cls(infs, sups, lies, width, depth, 0 if resolution is None else resolution,
                   support, device)

    def _query(self, infs, sups, resolution, logsig=True, sig=False):
        infs = np.ascontiguousarray(infs, dtype=np.float64).reshape(-1)
        sups = np.ascontiguousarray(sups, dtype=np.float64).reshape(-1)
        n = infs.shape[0]
        L, T = self.lie_basis.size(), self.tensor_basis.size()
        lie = torch.empty((n, L), dtype=torch.float64, device=self.device) if logsig else None
        sg = torch.empty((n, T), dtype=torch.float64, device=self.device) if sig else None
        if n == 0:
            return lie, sg
        res = _lib.QUERY_RESOLUTION_AUTO if resolution is None else int(resolution)
        npc = int(self.piece_inf.shape[0])
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib.rpyb_piecewise_query(
                self.width, self.depth, npc, self.piece_inf.ctypes.data if npc else None,
                self.piece_sup.ctypes.data if npc else None,
                self.pieces.data_ptr() if npc else None, L, float(self.support.inf),
                float(self.support.sup), self.resolution, n, infs.ctypes.data, sups.ctypes.data,
                res, lie.data_ptr() if logsig else None, L, sg.data_ptr() if sig else None, T,
                torch.cuda.current_stream(self.device).cuda_stream))
        return lie, sg


def sig_derivative_batch(logsigs, perturbations, offsets, width: int, depth: int,
                         device="cuda") -> torch.Tensor:
    """Forward-mode signature derivatives of many lists at once
    (``rpyb_sig_derivative``): list q is the pairs ``offsets[q]:offsets[q+1]``
    of rows of ``logsigs`` and ``perturbations`` (Hall coordinates).  The
    float64 or float32 dtype of ``logsigs`` is kept.  Returns ``[n_lists, T]``.
    Replaces Context::sig_derivative (algebra/src/lite_context.h:577-636)."""
    dev = torch.device(device)
    lg = torch.as_tensor(np.asarray(logsigs) if not torch.is_tensor(logsigs) else logsigs)
    dt = torch.float32 if lg.dtype == torch.float32 else torch.float64
    lg = lg.to(dev, dt).contiguous()
    pt = torch.as_tensor(np.asarray(perturbations) if not torch.is_tensor(perturbations)
                         else perturbations).to(dev, dt).contiguous()
    L = rpc.LieBasis(width, depth).size()
    T = rpc.TensorBasis(width, depth).size()
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    n = off.shape[0] - 1
    n_items = int(off[-1])
    if lg.dim() != 2 or lg.shape != pt.shape or lg.shape[0] != n_items or lg.shape[1] != L:
        raise ValueError("logsigs and perturbations must be [items, lie_dim] matching offsets")
    code = _lib.F64 if dt == torch.float64 else _lib.F32
    out = torch.empty((n, T), dtype=dt, device=dev)
    ws_n = int(_lib.lib.rpyb_sig_derivative_workspace_size(code, width, depth, n, n_items))
    if ws_n < 0:
        raise ValueError(_lib.last_error())
    ws = torch.empty(max(ws_n, 1), dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        _lib.check(_lib.lib.rpyb_sig_derivative(
            code, width, depth, n, off.ctypes.data, lg.data_ptr() if n_items else None,
            pt.data_ptr() if n_items else None, L, out.data_ptr(), T, ws.data_ptr(), ws.numel(),
            torch.cuda.current_stream(dev).cuda_stream))
    return out


def sig_derivative(pairs, width: int, depth: int, device="cuda") -> np.ndarray:
    """Derivative of the signature along the perturbations of one list of
    (log-signature, perturbation) pairs, as Context::sig_derivative computes
    it; float64 numpy result."""
    pairs = list(pairs)
    L = rpc.LieBasis(width, depth).size()
    lg = np.zeros((len(pairs), L))
    pt = np.zeros((len(pairs), L))
    for i, (x, p) in enumerate(pairs):
        x = np.asarray(x, dtype=np.float64).reshape(-1)
        p = np.asarray(p, dtype=np.float64).reshape(-1)
        lg[i, :min(L, x.size)] = x[:L]
        pt[i, :min(L, p.size)] = p[:L]
    out = sig_derivative_batch(lg, pt, [0, len(pairs)], width, depth, device)
    return out[0].cpu().numpy()


def cbh_batch(lies, offsets, width: int, depth: int, device="cuda") -> torch.Tensor:
    """Campbell-Baker-Hausdorff products of many lists of Lie elements
    (``rpyb_cbh``): list q holds rows ``offsets[q]:offsets[q+1]`` of ``lies``
    (Hall coordinates, [items, c] with c <= the Lie dimension).  Returns a
    float64 device tensor [n_lists, lie_dim]; row q is Context::cbh of the
    list (algebra/src/context.cpp:187-208)."""
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    L = rpc.LieBasis(width, depth).size()
    rows = np.asarray(lies, dtype=np.float64).reshape(-1, np.shape(lies)[-1] if np.ndim(lies) > 1
                                                       else L)
    full = np.zeros((rows.shape[0], L))
    full[:, :min(L, rows.shape[1])] = rows[:, :L]
    n = off.shape[0] - 1
    dev = torch.device(device)
    out = torch.zeros((n, L), dtype=torch.float64, device=dev)
    if n == 0:
        return out
    x = torch.from_numpy(full).to(dev)
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib.rpyb_cbh(int(width), int(depth), n, off.ctypes.data,
                                     x.data_ptr() if rows.shape[0] else None, L, out.data_ptr(),
                                     L, stream))
    return out


def cbh(lies, width: int, depth: int, device="cuda") -> np.ndarray:
    """Context::cbh of one sequence of Lie elements (Hall coordinates)."""
    rows = [np.asarray(x, dtype=np.float64).reshape(-1) for x in lies]
    L = rpc.LieBasis(width, depth).size()
    mat = np.zeros((len(rows), L))
    for i, r in enumerate(rows):
        mat[i, :min(L, r.size)] = r[:L]
    return cbh_batch(mat, [0, len(rows)], width, depth, device)[0].cpu().numpy()


class _DyadicTree:
    """Owner of an rpyb_dyadic_tree handle (device memory freed with it)."""

    def __init__(self, handle, device):
        self.handle = handle
        self.device = device
        self.range_table = False
        self.refresh()

    def refresh(self):
        """Re-read the node table's size and address (the range table moves it)."""
        rows = ctypes.c_int64()
        top = ctypes.c_int32()
        nodes = ctypes.c_void_p()
        _lib.check(_lib.lib.rpyb_dyadic_tree_info(self.handle, ctypes.byref(rows),
                                                  ctypes.byref(top), ctypes.byref(nodes)))
        self.rows, self.top_level, self.nodes = rows.value, top.value, nodes.value

    def node_row(self, level: int, block: int) -> int:
        return int(_lib.lib.rpyb_dyadic_node_row(self.handle, int(level), int(block)))

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h is not None and h.value:
            try:
                torch.cuda.current_stream(self.device).synchronize()
                _lib.lib.rpyb_dyadic_free(h)
            except Exception:
                pass

