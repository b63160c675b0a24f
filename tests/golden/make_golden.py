"""Generate the golden fixtures in this directory from the reference itself.

Run in a container that has the RoughPy sources (``make -C oracle ref``
builds the reference ``roughpy.compute`` extension from them into
``oracle/_ref``):

    python tests/golden/make_golden.py

Every expected array below is computed by the reference's own compiled
``roughpy.compute`` (float64 unless stated), on seeded synthetic inputs.
The fixtures are committed so that the tests need neither the reference
sources nor the reference build.
"""
from __future__ import annotations

import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

rpc = oracle.ref_compute()
if rpc is None:
    raise SystemExit("reference build missing: run `make -C oracle ref` first")


def level_scaled(rng, width, depth, batch, unit=True):
    """Level-0 coefficient 1 and level-k coefficients N(0,1)/k!."""
    basis = rpc.TensorBasis(width, depth)
    db = basis.degree_begin
    x = np.zeros((batch, basis.size()))
    fact = 1.0
    for k in range(depth + 1):
        if k > 0:
            fact *= k
        x[:, db[k]:db[k + 1]] = rng.standard_normal((batch, db[k + 1] - db[k])) / fact
    if unit:
        x[:, 0] = 1.0
    return x


def ft(data, basis):
    return rpc.FreeTensor(data, basis)


def gen_tensor_ops():
    out = {}
    rng = np.random.default_rng(20240501)
    # reference known answer (tests/compute/test_ft_fma.py:7-20), float32
    basis = rpc.TensorBasis(2, 2)
    b = np.array([2, 1, 3, 0.5, -1, 2, 0], dtype=np.float32)
    c = np.array([-1, 4, 0, 1, 1, 0, 2], dtype=np.float32)
    a = ft(np.zeros(basis.size(), dtype=np.float32), basis)
    rpc.ft_fma(a, ft(b, basis), ft(c, basis))
    out["fma_explicit_b"] = b
    out["fma_explicit_c"] = c
    out["fma_explicit_out"] = a.data

    cases = [(2, 4), (3, 3), (4, 3), (2, 6), (5, 2)]
    for (w, d) in cases:
        basis = rpc.TensorBasis(w, d)
        tag = f"w{w}d{d}"
        A = level_scaled(rng, w, d, 3)
        B = level_scaled(rng, w, d, 3)
        C = level_scaled(rng, w, d, 3)
        out[f"{tag}_A"], out[f"{tag}_B"], out[f"{tag}_C"] = A, B, C
        # fma with every combination of depth truncations the bindings expose
        for (od, ld, rd) in [(-1, -1, -1), (d - 1, -1, -1), (-1, d - 1, -1), (-1, -1, 1),
                             (2, 1, 1)]:
            res = A.copy()
            rpc._internals.dense_ft_fma(res, B, C, basis, od, ld, rd)
            out[f"{tag}_fma_{od}_{ld}_{rd}"] = res
        # in-place multiply with and without a truncated rhs
        for (od, rd) in [(-1, -1), (-1, 1), (d - 1, -1)]:
            res = B.copy()
            rpc._internals.dense_ft_inplace_mul(res, C, basis, od, rd)
            out[f"{tag}_imul_{od}_{rd}"] = res
        # exp / fmexp of level-1+ arguments, log of group-like elements
        X = level_scaled(rng, w, d, 3, unit=False)
        X[:, 0] = 0.0
        out[f"{tag}_X"] = X
        out[f"{tag}_exp"] = rpc.ft_exp(ft(X, basis)).data
        out[f"{tag}_fmexp"] = rpc.ft_fmexp(ft(A, basis), ft(X, basis)).data
        E = out[f"{tag}_exp"]
        out[f"{tag}_log"] = rpc.ft_log(ft(E, basis)).data
        out[f"{tag}_log_A"] = rpc.ft_log(ft(A, basis)).data
        out[f"{tag}_antipode"] = rpc.antipode(ft(A, basis)).data
        adj = np.zeros_like(C)
        rpc._internals.dense_ft_adjoint_left_mul(adj, B, C, basis, d, d, d)
        out[f"{tag}_adjlmul"] = adj
        # float32 copies for the dtype path of the bindings
        A32 = A.astype(np.float32)
        B32 = B.astype(np.float32)
        C32 = C.astype(np.float32)
        res = A32.copy()
        rpc._internals.dense_ft_fma(res, B32, C32, basis)
        out[f"{tag}_fma32"] = res
        out[f"{tag}_exp32"] = rpc.ft_exp(ft(X.astype(np.float32), basis)).data
    return out


def gen_lie():
    out = {}
    rng = np.random.default_rng(7)
    for (w, d) in [(2, 4), (3, 4), (4, 5), (6, 5), (8, 5), (5, 4)]:
        lb = rpc.LieBasis(w, d)
        tb = rpc.TensorBasis(w, d)
        tag = f"w{w}d{d}"
        out[f"{tag}_data"] = np.asarray(lb.data, dtype=np.int64)
        out[f"{tag}_degree_begin"] = np.asarray(lb.degree_begin, dtype=np.int64)
        # pin both maps on seeded random vectors (size-independent check)
        rows = 3 if tb.size() < 5000 else 1
        L = rng.standard_normal((rows, lb.size()))
        Tn = rng.standard_normal((rows, tb.size()))
        out[f"{tag}_l2t_in"] = L
        out[f"{tag}_l2t_out"] = rpc.lie_to_tensor(rpc.Lie(L, lb), tb).data
        out[f"{tag}_t2l_in"] = Tn
        out[f"{tag}_t2l_out"] = rpc.tensor_to_lie(rpc.FreeTensor(Tn, tb), lb).data
    # full maps as dense matrices for small shapes
    for (w, d) in [(2, 4), (3, 3), (4, 3)]:
        lb = rpc.LieBasis(w, d)
        tb = rpc.TensorBasis(w, d)
        tag = f"w{w}d{d}"
        eye_l = np.eye(lb.size())
        eye_t = np.eye(tb.size())
        out[f"{tag}_l2t_dense"] = rpc.lie_to_tensor(rpc.Lie(eye_l, lb), tb).data.T.copy()
        out[f"{tag}_t2l_dense"] = rpc.tensor_to_lie(rpc.FreeTensor(eye_t, tb), lb).data.T.copy()
    return out


def fmexp_chain(width, depth, inc):
    """Reference signature of one stream: chained ft_fmexp (the survey's recipe)."""
    basis = rpc.TensorBasis(width, depth)
    sig = np.zeros(basis.size())
    sig[0] = 1.0
    x = np.zeros(basis.size())
    for row in inc:
        x[1:1 + width] = row
        sig = rpc.ft_fmexp(ft(sig, basis), ft(x, basis)).data
    return sig


def gen_signatures():
    out = {}
    rng = np.random.default_rng(0)
    for (w, d, lens) in [(4, 5, [128, 1, 37, 0, 5]), (2, 6, [64, 3]), (3, 4, [50, 17]),
                         (8, 3, [40, 9]), (5, 4, [33]), (8, 5, [24, 3])]:
        tag = f"w{w}d{d}"
        off = np.zeros(len(lens) + 1, dtype=np.int64)
        off[1:] = np.cumsum(lens)
        inc = rng.normal(0.0, np.sqrt(1.0 / 128), size=(int(off[-1]), w))
        out[f"{tag}_offsets"] = off
        out[f"{tag}_inc"] = inc
        out[f"{tag}_sig"] = np.stack([fmexp_chain(w, d, inc[off[s]:off[s + 1]])
                                      for s in range(len(lens))])
    return out


def ref_arith(width, depth):
    """Stream restatement arithmetic backed by the reference roughpy.compute."""
    from oracle.streams_ref import Arith
    tb = rpc.TensorBasis(width, depth)
    lb = rpc.LieBasis(width, depth)
    l2t = rpc.lie_to_tensor(rpc.Lie(np.eye(lb.size()), lb), tb).data.T.copy()
    t2l = rpc.tensor_to_lie(rpc.FreeTensor(np.eye(tb.size()), tb), lb).data.T.copy()
    return Arith(width, depth, l2t, t2l,
                 lambda x: rpc.ft_exp(ft(np.asarray(x, dtype=np.float64), tb)).data,
                 lambda a, x: rpc.ft_fmexp(ft(np.asarray(a, dtype=np.float64), tb),
                                           ft(np.asarray(x, dtype=np.float64), tb)).data,
                 lambda x: rpc.ft_log(ft(np.asarray(x, dtype=np.float64), tb)).data)


def gen_streams():
    """Stream queries through the restated DyadicCachingLayer, reference arithmetic."""
    from oracle.streams_ref import StreamRef
    out = {}
    rng = np.random.default_rng(3)
    cases = [
        ("a", 2, 3, 40, None, None),      # default indices (resolution 0)
        ("b", 3, 3, 64, "grid", 6),       # events on a 2^-6 grid, explicit resolution
        ("c", 2, 4, 30, "random", None),  # random times, heuristic resolution
        ("d", 3, 2, 25, "random", 3),     # coarse resolution: several events per leaf
    ]
    for tag, w, d, n, kind, res in cases:
        ar = ref_arith(w, d)
        inc = rng.normal(0, 0.3, size=(n, w))
        if kind is None:
            idx = None
        elif kind == "grid":
            idx = np.arange(n) / 64.0
        else:
            idx = np.sort(rng.uniform(0.0, 2.0, size=n))
        st = StreamRef(ar, inc, idx, res)
        s0, s1 = st.support
        qs = [(s0, s1), (s0 - 1.0, s0), (s0 + 0.3 * (s1 - s0), s0 + 0.3 * (s1 - s0)),
              (s1 + 0.5, s1 + 1.0)]
        for _ in range(14):
            a, b = np.sort(rng.uniform(s0 - 0.2, s1 + 0.2, size=2))
            qs.append((float(a), float(b)))
        qs = np.array(qs)
        out[f"{tag}_inc"] = inc
        out[f"{tag}_idx"] = np.array([]) if idx is None else idx
        out[f"{tag}_meta"] = np.array([w, d, -1 if res is None else res])
        out[f"{tag}_queries"] = qs
        out[f"{tag}_resolution"] = np.array([st.resolution])
        out[f"{tag}_logsig"] = np.stack([st.log_signature(a, b) for a, b in qs])
        out[f"{tag}_sig"] = np.stack([st.signature(a, b) for a, b in qs])
    return out


if __name__ == "__main__":
    np.savez_compressed(HERE / "tensor_ops.npz", **gen_tensor_ops())
    np.savez_compressed(HERE / "lie_maps.npz", **gen_lie())
    np.savez_compressed(HERE / "signatures.npz", **gen_signatures())
    np.savez_compressed(HERE / "streams.npz", **gen_streams())
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)
