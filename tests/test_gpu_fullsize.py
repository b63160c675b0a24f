"""Parity at the benchmark's full sizes.

* Uneven batched signatures: 4096 streams with lengths uniform in [16, 4096],
  width 8, depth 5, increments N(0, 1/len) (the headline workload, seed 2):
  the float32 path against the float64 path on the same inputs <= 1e-6 per
  level, the float64 path against the C oracle on 16 of the streams (the
  longest among them) <= 1e-12, and the per-stream error report equal to the
  comparison.
* Long streams: 8 streams of 16384 increments.
* Dyadic-cache queries: 2^16 events at t_i = i 2^-16, width 6, depth 5,
  resolution 16 (seed 3): a float32 tree against the float64 tree on 2000 of
  the 100000 query intervals <= 1e-6, and short queries against the
  restated DyadicCachingLayer <= 1e-12.
"""
import numpy as np
import pytest
import torch

import oracle
from roughpy_b200 import signatures as S
from tests._util import level_rel_err

pytestmark = pytest.mark.gpu

WIDTH, DEPTH = 8, 5


def uneven_workload(seed=2, n=4096, lo=16, hi=4096):
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, size=n)
    off = S.offsets_from_lengths(lens)
    inc = np.empty((int(off[-1]), WIDTH), dtype=np.float32)
    for s in range(n):
        L = int(lens[s])
        inc[off[s]:off[s + 1]] = rng.normal(0.0, np.sqrt(1.0 / L), size=(L, WIDTH))
    return lens, off, inc


def level_err_rows(got, want, width, depth):
    """Per-row per-level relative error on the device (float64)."""
    db = [0]
    for _ in range(depth + 1):
        db.append(1 + width * db[-1])
    worst = torch.zeros(got.shape[0], dtype=torch.float64, device=got.device)
    g = got.double()
    for k in range(depth + 1):
        a, b = g[:, db[k]:db[k + 1]], want[:, db[k]:db[k + 1]]
        num = (a - b).abs().amax(dim=1)
        den = b.abs().amax(dim=1)
        worst = torch.maximum(worst, torch.where(den > 0, num / den.clamp_min(1e-300), num))
    return worst


@pytest.fixture(scope="module")
def config3():
    lens, off, inc = uneven_workload()
    x32 = torch.from_numpy(inc).cuda()
    p32 = S.SignaturePlan(off, WIDTH, DEPTH, "f32c")
    p64 = S.SignaturePlan(off, WIDTH, DEPTH, "f64")
    out32, err = p32.run(x32, report_error=True)
    out64 = p64.run(x32.double())
    torch.cuda.synchronize()
    return lens, off, inc, out32, out64, err


def test_uneven_float32_against_float64_full_batch(config3):
    lens, off, inc, out32, out64, err = config3
    rows = level_err_rows(out32, out64, WIDTH, DEPTH)
    assert float(rows.max()) <= 1e-6, float(rows.max())
    # the report of rpyb_sig_plan_run is the same comparison
    assert float((rows - err).abs().max()) <= 1e-12


def test_uneven_float64_against_oracle_sample(config3):
    lens, off, inc, out32, out64, err = config3
    rng = np.random.default_rng(17)
    idx = np.concatenate([[int(np.argmax(lens))], rng.choice(len(lens), size=15, replace=False)])
    got = out64.cpu().numpy()
    for s in idx:
        rows = inc[off[s]:off[s + 1]].astype(np.float64)
        want = oracle.signature(WIDTH, DEPTH, rows)
        assert level_rel_err(got[s], want, WIDTH, DEPTH) <= 1e-12, s


def test_long_streams_float32_against_float64():
    rng = np.random.default_rng(5)
    n, L = 8, 16384
    off = np.arange(n + 1, dtype=np.int64) * L
    inc = rng.normal(0.0, np.sqrt(1.0 / L), size=(n * L, WIDTH)).astype(np.float32)
    x = torch.from_numpy(inc).cuda()
    out32 = S.SignaturePlan(off, WIDTH, DEPTH, "f32c").run(x)
    out64 = S.SignaturePlan(off, WIDTH, DEPTH, "f64").run(x.double())
    torch.cuda.synchronize()
    err = float(level_err_rows(out32, out64, WIDTH, DEPTH).max())
    assert err <= 1e-6, err
    want = oracle.signature(WIDTH, DEPTH, inc[:L].astype(np.float64))
    assert level_rel_err(out64[0].cpu().numpy(), want, WIDTH, DEPTH) <= 1e-12


def dense_lie_map(w, d, which):
    """rpyb_lie_map_csr as a dense float64 matrix (0: l2t, 1: t2l)."""
    import ctypes
    from roughpy_b200 import _lib
    nnz = int(_lib.lib.rpyb_lie_map_csr(w, d, which, None, None, None))
    T = int(_lib.lib.rpyb_tensor_size(w, d))
    L = int(_lib.lib.rpyb_lie_basis_size(w, d))
    rows, cols = (T, L) if which == 0 else (L, T)
    indptr = np.zeros(rows + 1, dtype=np.int64)
    indices = np.zeros(nnz, dtype=np.int64)
    values = np.zeros(nnz, dtype=np.float64)
    p64 = ctypes.POINTER(ctypes.c_int64)
    pd = ctypes.POINTER(ctypes.c_double)
    rc = _lib.lib.rpyb_lie_map_csr(w, d, which, indptr.ctypes.data_as(p64),
                                   indices.ctypes.data_as(p64), values.ctypes.data_as(pd))
    assert rc >= 0
    dense = np.zeros((rows, cols))
    for r in range(rows):
        dense[r, indices[indptr[r]:indptr[r + 1]]] = values[indptr[r]:indptr[r + 1]]
    return dense


@pytest.fixture(scope="module")
def dyadic_stream():
    from roughpy_b200.streams import LieIncrementStream
    n = 1 << 16
    rng = np.random.default_rng(3)
    inc = rng.normal(0, np.sqrt(1.0 / n), size=(n, 6))
    idx = np.arange(n) / n
    q = np.sort(np.floor(rng.uniform(0, 1, size=(100000, 2)) * n) / n, axis=1)
    inc32 = inc.astype(np.float32)
    s32 = LieIncrementStream.from_increments(inc32, indices=idx, width=6, depth=5, resolution=16)
    s64 = LieIncrementStream.from_increments(inc32.astype(np.float64), indices=idx, width=6,
                                             depth=5, resolution=16)
    return inc32.astype(np.float64), idx, q, s32, s64


def test_dyadic_full_size_float32_tree_against_float64_tree(dyadic_stream):
    inc, idx, q, s32, s64 = dyadic_stream
    assert s32.mode == "f32c" and s64.mode == "f64"
    sample = q[np.random.default_rng(1).choice(q.shape[0], size=2000, replace=False)]
    got = s32.signature_batch(sample[:, 0], sample[:, 1]).cpu().numpy()
    want = s64.signature_batch(sample[:, 0], sample[:, 1]).cpu().numpy()
    assert level_rel_err(got, want, 6, 5) <= 1e-6
    lie32 = s32.log_signature_batch(sample[:, 0], sample[:, 1]).cpu().numpy()
    lie64 = s64.log_signature_batch(sample[:, 0], sample[:, 1]).cpu().numpy()
    scale = np.maximum(np.abs(lie64).max(axis=1, keepdims=True), 1e-300)
    assert float((np.abs(lie32 - lie64) / scale).max()) <= 1e-6
    # the whole support is the Chen product of every increment
    full = s64.signature(0.0, 1.0)
    assert level_rel_err(full, oracle.signature(6, 5, inc), 6, 5) <= 1e-11


def test_dyadic_full_size_short_queries_against_restatement(dyadic_stream):
    from oracle import streams_ref as R
    inc, idx, q, s32, s64 = dyadic_stream
    w, d = 6, 5
    # dense maps from the library's CSR maps (equal to the reference's maps:
    # tests/test_gpu_tensor_ops.py and tests/test_lie_host.py)
    l2t, t2l = dense_lie_map(w, d, 0), dense_lie_map(w, d, 1)
    ref = R.StreamRef(R.Arith.from_oracle(w, d, l2t, t2l), inc, idx, 16)
    n = 1 << 16
    rng = np.random.default_rng(9)
    a = rng.integers(0, n - 40, size=5)
    b = a + rng.integers(1, 40, size=5)
    qs = np.stack([a / n, b / n], axis=1)
    got = s64.signature_batch(qs[:, 0], qs[:, 1]).cpu().numpy()
    want = np.stack([ref.signature(x, y) for x, y in qs])
    assert level_rel_err(got, want, w, d) <= 1e-12
