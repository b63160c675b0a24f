"""GPU parity of the dense free-tensor operations (roughpy_b200.compute and the
C ABI behind it) against the reference's outputs and the CPU oracle.

Tolerances (per-level normwise relative error, tests/_util.level_rel_err):
float64 <= 1e-12; float32 rows (compensated accumulation) <= 2e-6 against the
float64 oracle evaluated on the same float32 inputs.
"""
import numpy as np
import pytest
import torch

import oracle
from roughpy_b200 import _internals as I
from roughpy_b200 import compute as rpc
from tests._util import level_rel_err, level_scaled

pytestmark = pytest.mark.gpu

CASES = [(2, 4), (3, 3), (4, 3), (2, 6), (5, 2)]
F64_TOL = 1e-12
F32_TOL = 2e-6


def test_fma_explicit_known_answer(golden):
    # tests/compute/test_ft_fma.py:7-20 through the public API, float32
    g = golden["tensor_ops"]
    basis = rpc.TensorBasis(2, 2)
    a = rpc.FreeTensor(np.zeros(basis.size(), dtype=np.float32), basis)
    rpc.ft_fma(a, rpc.FreeTensor(g["fma_explicit_b"], basis),
               rpc.FreeTensor(g["fma_explicit_c"], basis))
    np.testing.assert_array_equal(a.data, g["fma_explicit_out"])


def test_exp_letter_and_log_identity_exact():
    basis = rpc.TensorBasis(2, 2)
    e = rpc.ft_exp(rpc.FreeTensor(np.array([0.0, 1, 0, 0, 0, 0, 0]), basis))
    np.testing.assert_array_equal(e.data, [1.0, 1.0, 0.0, 0.5, 0.0, 0.0, 0.0])
    z = rpc.ft_exp(rpc.FreeTensor(np.zeros(7), basis))
    np.testing.assert_array_equal(z.data, [1.0, 0, 0, 0, 0, 0, 0])
    lg = rpc.ft_log(rpc.FreeTensor(np.array([1.0, 0, 0, 0, 0, 0, 0]), basis))
    np.testing.assert_array_equal(lg.data, np.zeros(7))


@pytest.mark.parametrize("w,d", CASES)
def test_fma_against_reference_with_bounds(golden, w, d):
    g = golden["tensor_ops"]
    t = f"w{w}d{d}"
    basis = rpc.TensorBasis(w, d)
    for (od, ld, rd) in [(-1, -1, -1), (d - 1, -1, -1), (-1, d - 1, -1), (-1, -1, 1), (2, 1, 1)]:
        res = g[f"{t}_A"].copy()
        I.dense_ft_fma(res, g[f"{t}_B"], g[f"{t}_C"], basis, od, ld, rd)
        assert level_rel_err(res, g[f"{t}_fma_{od}_{ld}_{rd}"], w, d) <= F64_TOL, (od, ld, rd)
    res = g[f"{t}_A"].astype(np.float32)
    I.dense_ft_fma(res, g[f"{t}_B"].astype(np.float32), g[f"{t}_C"].astype(np.float32), basis)
    want = oracle.ft_fma(w, d, g[f"{t}_A"].astype(np.float32), g[f"{t}_B"].astype(np.float32),
                         g[f"{t}_C"].astype(np.float32))
    assert level_rel_err(res, want, w, d) <= F32_TOL
    assert level_rel_err(res, g[f"{t}_fma32"], w, d) <= F32_TOL


@pytest.mark.parametrize("w,d", CASES)
def test_inplace_mul_against_reference(golden, w, d):
    g = golden["tensor_ops"]
    t = f"w{w}d{d}"
    basis = rpc.TensorBasis(w, d)
    for (od, rd) in [(-1, -1), (-1, 1), (d - 1, -1)]:
        res = g[f"{t}_B"].copy()
        I.dense_ft_inplace_mul(res, g[f"{t}_C"], basis, od, rd)
        assert level_rel_err(res, g[f"{t}_imul_{od}_{rd}"], w, d) <= F64_TOL


@pytest.mark.parametrize("w,d", CASES)
def test_series_against_reference(golden, w, d):
    g = golden["tensor_ops"]
    t = f"w{w}d{d}"
    basis = rpc.TensorBasis(w, d)
    X, A = g[f"{t}_X"], g[f"{t}_A"]
    assert level_rel_err(rpc.ft_exp(rpc.FreeTensor(X, basis)).data, g[f"{t}_exp"], w, d) <= F64_TOL
    got = rpc.ft_fmexp(rpc.FreeTensor(A, basis), rpc.FreeTensor(X, basis)).data
    assert level_rel_err(got, g[f"{t}_fmexp"], w, d) <= F64_TOL
    got = rpc.ft_log(rpc.FreeTensor(g[f"{t}_exp"], basis)).data
    assert level_rel_err(got, g[f"{t}_log"], w, d) <= 1e-11
    got = rpc.ft_log(rpc.FreeTensor(A, basis)).data
    assert level_rel_err(got, g[f"{t}_log_A"], w, d) <= 1e-11
    got = rpc.antipode(rpc.FreeTensor(A, basis)).data
    np.testing.assert_array_equal(got, g[f"{t}_antipode"])
    got = rpc.ft_adjoint_left_mul(rpc.FreeTensor(g[f"{t}_B"], basis),
                                  rpc.ShuffleTensor(g[f"{t}_C"], basis)).data
    assert level_rel_err(got, g[f"{t}_adjlmul"], w, d) <= F64_TOL
    got32 = rpc.ft_exp(rpc.FreeTensor(X.astype(np.float32), basis)).data
    assert got32.dtype == np.float32
    assert level_rel_err(got32, g[f"{t}_exp32"], w, d) <= F32_TOL


@pytest.mark.parametrize("w,d,batch", [(2, 12, 5), (4, 8, 3), (6, 6, 2), (8, 6, 2), (8, 5, 7),
                                       (3, 7, 4), (7, 4, 3), (9, 3, 2)])
def test_fma_sweep_shapes_against_oracle(w, d, batch):
    """The FMA sweep shapes (level k ~ N(0,1)/k!, unit level 0), both dtypes."""
    rng = np.random.default_rng(1 + w * 100 + d)
    A = level_scaled(rng, w, d, batch)
    B = level_scaled(rng, w, d, batch)
    C = level_scaled(rng, w, d, batch)
    want = oracle.ft_fma(w, d, A, B, C)
    basis = rpc.TensorBasis(w, d)
    got = A.copy()
    I.dense_ft_fma(got, B, C, basis)
    assert level_rel_err(got, want, w, d) <= F64_TOL
    A32, B32, C32 = (x.astype(np.float32) for x in (A, B, C))
    want32 = oracle.ft_fma(w, d, A32, B32, C32)
    got32 = A32.copy()
    I.dense_ft_fma(got32, B32, C32, basis)
    assert level_rel_err(got32, want32, w, d) <= F32_TOL


def test_torch_inputs_in_place_and_batch_dims():
    w, d = 3, 4
    rng = np.random.default_rng(3)
    A = level_scaled(rng, w, d, 6).reshape(2, 3, -1)
    B = level_scaled(rng, w, d, 6).reshape(2, 3, -1)
    C = level_scaled(rng, w, d, 6).reshape(2, 3, -1)
    want = oracle.ft_fma(w, d, A, B, C)
    ta = torch.from_numpy(A).cuda()
    ptr = ta.data_ptr()
    I.dense_ft_fma(ta, torch.from_numpy(B).cuda(), torch.from_numpy(C).cuda(),
                   rpc.TensorBasis(w, d))
    assert ta.data_ptr() == ptr
    assert level_rel_err(ta.cpu().numpy(), want, w, d) <= F64_TOL


def test_mismatched_arguments_raise():
    basis = rpc.TensorBasis(2, 2)
    with pytest.raises(TypeError):
        I.dense_ft_fma(np.zeros(7), np.zeros(7, dtype=np.float32), np.zeros(7), basis)
    with pytest.raises(ValueError):
        I.dense_ft_fma(np.zeros((2, 7)), np.zeros((3, 7)), np.zeros((2, 7)), basis)


@pytest.mark.parametrize("w,d", [(2, 5), (4, 4), (5, 3)])
def test_exp_log_roundtrip_and_gather(w, d):
    rng = np.random.default_rng(11)
    basis = rpc.TensorBasis(w, d)
    x = np.zeros((4, basis.size()))
    x[:, 1:1 + w] = rng.normal(size=(4, w))
    e = rpc.ft_exp(rpc.FreeTensor(x, basis))
    back = rpc.ft_log(e)
    np.testing.assert_array_almost_equal(back.data, x, decimal=13)
    # gathered product rows: out[i] = lhs[li[i]] * rhs[ri[i]]
    from roughpy_b200 import _lib
    rows = torch.from_numpy(e.data).cuda()
    out = torch.zeros_like(rows)
    li = torch.tensor([3, 0, 1, 2], device="cuda")
    ri = torch.tensor([1, 1, 0, 3], device="cuda")
    _lib.check(_lib.lib.rpyb_ft_mul_gather(_lib.F64, w, d, 4, out.data_ptr(), rows.data_ptr(),
                                           rows.data_ptr(), basis.size(), None, li.data_ptr(),
                                           ri.data_ptr(), 0, 0))
    torch.cuda.synchronize()
    want = oracle.ft_mul(w, d, e.data[[3, 0, 1, 2]], e.data[[1, 1, 0, 3]])
    assert level_rel_err(out.cpu().numpy(), want, w, d) <= F64_TOL


def test_lie_maps_on_gpu(golden):
    g = golden["lie_maps"]
    for (w, d) in [(2, 4), (4, 5), (6, 5), (8, 5)]:
        t = f"w{w}d{d}"
        lb = rpc.LieBasis(w, d)
        tb = rpc.TensorBasis(w, d)
        got = rpc.lie_to_tensor(rpc.Lie(g[f"{t}_l2t_in"], lb), tb).data
        np.testing.assert_allclose(got, g[f"{t}_l2t_out"], rtol=0, atol=1e-12)
        got = rpc.tensor_to_lie(rpc.FreeTensor(g[f"{t}_t2l_in"], tb), lb).data
        np.testing.assert_allclose(got, g[f"{t}_t2l_out"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("w,d", [(4, 4), (3, 5), (8, 3), (6, 5)])
def test_c_abi_tensor_lie_maps(w, d):
    """rpyb_tensor_to_lie / rpyb_lie_to_tensor (device-cached maps, assigning
    outputs) equal the roughpy.compute-style dense maps, and t2l(l2t(x)) = x
    on Lie elements; float32 rows within 1e-6."""
    import torch
    from roughpy_b200 import _lib
    from roughpy_b200 import compute as rpc
    lb, tb = rpc.LieBasis(w, d), rpc.TensorBasis(w, d)
    L, T = lb.size(), tb.size()
    rng = np.random.default_rng(w * 5 + d)
    x = torch.from_numpy(rng.normal(size=(7, L))).cuda()
    emb = torch.full((7, T), 3.0, dtype=torch.float64, device="cuda")   # overwritten
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib.rpyb_lie_to_tensor(_lib.F64, w, d, 7, emb.data_ptr(), T, x.data_ptr(), L, s))
    want = torch.zeros((7, T), dtype=torch.float64, device="cuda")
    rpc._internals.dense_lie_to_tensor(want, x, lb.get_l2t_matrix(), lb, tb)
    assert float((emb - want).abs().max()) <= 1e-14 * float(want.abs().max())
    back = torch.full((7, L), -1.0, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib.rpyb_tensor_to_lie(_lib.F64, w, d, 7, back.data_ptr(), L, emb.data_ptr(), T,
                                           s))
    assert float((back - x).abs().max()) <= 1e-13 * float(x.abs().max())
    nb = 300   # more rows than blocks: each block projects several
    t = torch.from_numpy(rng.normal(size=(nb, T))).cuda()
    got = torch.empty((nb, L), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib.rpyb_tensor_to_lie(_lib.F64, w, d, nb, got.data_ptr(), L, t.data_ptr(), T,
                                           s))
    ref = torch.zeros((nb, L), dtype=torch.float64, device="cuda")
    rpc._internals.dense_tensor_to_lie(ref, t, lb.get_t2l_matrix(), lb, tb)
    assert float((got - ref).abs().max()) <= 1e-14 * float(ref.abs().max())
    t32 = t.float()
    got32 = torch.empty((nb, L), dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib.rpyb_tensor_to_lie(_lib.F32, w, d, nb, got32.data_ptr(), L, t32.data_ptr(),
                                           T, s))
    assert float((got32.double() - ref).abs().max()) <= 1e-6 * float(ref.abs().max())


@pytest.mark.parametrize("batch", [7, 300])
@pytest.mark.parametrize("n_rows,n_cols", [(97, 1500), (1960, 9331)])
def test_c_abi_sparse_map_accumulates_with_strides(batch, n_rows, n_cols):
    """rpyb_sparse_map, y += scale M x, in both dtypes, with row strides above
    the sizes; entries whose column lies outside [0, n_cols) are skipped.
    Checked against a float64 dense product."""
    from roughpy_b200 import _lib
    rng = np.random.default_rng(n_rows + batch)
    nnz_row = rng.integers(0, 20, size=n_rows)
    ptr = np.concatenate([[0], np.cumsum(nnz_row)]).astype(np.int64)
    idx = rng.integers(0, n_cols, size=int(ptr[-1])).astype(np.int64)
    val = rng.normal(size=int(ptr[-1]))
    bad = rng.random(idx.shape[0]) < 0.05
    idx[bad] = np.where(rng.random(int(bad.sum())) < 0.5, -1, n_cols)
    M = np.zeros((n_rows, n_cols))
    for r in range(n_rows):
        for k in range(ptr[r], ptr[r + 1]):
            if 0 <= idx[k] < n_cols:
                M[r, idx[k]] += val[k]
    x = rng.normal(size=(batch, n_cols + 5))
    y0 = rng.normal(size=(batch, n_rows + 3))
    d_ptr, d_idx, d_val = (torch.from_numpy(a).cuda() for a in (ptr, idx, val))
    s = torch.cuda.current_stream().cuda_stream
    for dt, code, tol in ((torch.float64, _lib.F64, 1e-12), (torch.float32, _lib.F32, 1e-5)):
        xd = torch.from_numpy(x).to(dt).cuda()
        yd = torch.from_numpy(y0).to(dt).cuda()
        _lib.check(_lib.lib.rpyb_sparse_map(code, n_rows, n_cols, batch, d_ptr.data_ptr(),
                                            d_idx.data_ptr(), d_val.data_ptr(), yd.data_ptr(),
                                            xd.data_ptr(), n_rows + 3, n_cols + 5, 0.5, s))
        torch.cuda.synchronize()
        got = yd.double().cpu().numpy()
        xr = xd.double().cpu().numpy()
        ref = torch.from_numpy(y0).to(dt).double().numpy()
        ref[:, :n_rows] += 0.5 * xr[:, :n_cols] @ M.T
        assert np.abs(got - ref).max() <= tol * max(1.0, np.abs(ref).max())
