"""GPU signature adjoint (reverse Chen products with checkpoint recomputation)
against float64 references: a differentiable float64 torch Chen product (exact
gradients by autograd), central finite differences (h = 1e-6) of the float64
signature kernel, and the float64 kernel's own gradient for the float32 mode.
Tolerances: float64 <= 1e-10 relative to the gradient's max magnitude against
autograd, <= 1e-6 against finite differences; float32 <= 1e-5."""
import numpy as np
import pytest
import torch

from roughpy_b200 import signatures as S

pytestmark = pytest.mark.gpu


def torch_signature(inc, width, depth):
    """Dense float64 Chen product of exp(x_t) written with torch ops (autograd)."""
    levels = [torch.ones(1, dtype=inc.dtype, device=inc.device)]
    for k in range(1, depth + 1):
        levels.append(torch.zeros(width ** k, dtype=inc.dtype, device=inc.device))
    for t in range(inc.shape[0]):
        x = inc[t]
        ex = [torch.ones(1, dtype=inc.dtype, device=inc.device)]
        for k in range(1, depth + 1):
            ex.append(torch.outer(ex[-1], x).reshape(-1) / k)
        new = []
        for k in range(depth + 1):
            acc = torch.zeros(width ** k, dtype=inc.dtype, device=inc.device)
            for j in range(k + 1):
                acc = acc + torch.outer(levels[k - j], ex[j]).reshape(-1)
            new.append(acc)
        levels = new
    return torch.cat(levels)


@pytest.mark.parametrize("w,d,lens,K", [(2, 3, [7, 1, 0, 12], 4), (3, 4, [20, 33], 64),
                                        (4, 3, [9, 16], 1), (5, 2, [11], 3),
                                        (2, 5, [9, 4, 70], 8), (3, 5, [6, 40], 16),
                                        (8, 5, [3, 5], 2), (2, 8, [5, 37], 64),
                                        (4, 6, [4, 1], 3), (6, 6, [3], 2), (3, 1, [5, 2], 2)])
def test_f64_gradient_equals_autograd(w, d, lens, K):
    rng = np.random.default_rng(w + 10 * d)
    off = S.offsets_from_lengths(lens)
    inc = torch.from_numpy(rng.normal(0, 0.4, size=(int(off[-1]), w))).cuda()
    T = S.tensor_size(w, d)
    W = torch.from_numpy(rng.normal(size=(len(lens), T))).cuda()
    plan = S.SignaturePlan(off, w, d, "f64")
    x = inc.clone().requires_grad_(True)
    sig = S.signature_with_grad(x, plan, checkpoint_every=K)
    (sig * W).sum().backward()
    got = x.grad
    xr = inc.clone().requires_grad_(True)
    loss = 0
    for s in range(len(lens)):
        loss = loss + (torch_signature(xr[off[s]:off[s + 1]], w, d) * W[s]).sum()
    loss.backward()
    want = xr.grad
    scale = float(want.abs().max()) if want.numel() else 1.0
    assert float((got - want).abs().max()) <= 1e-10 * max(scale, 1.0)
    ref_sig = torch.stack([torch_signature(inc[off[s]:off[s + 1]], w, d)
                           for s in range(len(lens))])
    assert float((sig.detach() - ref_sig).abs().max()) <= 1e-12 * float(ref_sig.abs().max())


@pytest.mark.parametrize("w,d", [(8, 5), (3, 5), (2, 2)])
def test_f32_gradient_against_f64(w, d):
    rng = np.random.default_rng(100 + w * d)
    lens = [50, 7, 130]
    off = S.offsets_from_lengths(lens)
    inc = torch.from_numpy(rng.normal(0, 0.2, size=(int(off[-1]), w))).cuda()
    T = S.tensor_size(w, d)
    W = torch.from_numpy(rng.normal(size=(len(lens), T))).cuda()
    x32 = inc.float().clone().requires_grad_(True)
    (S.signature_with_grad(x32, S.SignaturePlan(off, w, d, "f32c")).double() * W).sum().backward()
    x64 = inc.float().double().clone().requires_grad_(True)
    (S.signature_with_grad(x64, S.SignaturePlan(off, w, d, "f64")) * W).sum().backward()
    err = float((x32.grad.double() - x64.grad).abs().max()) / float(x64.grad.abs().max())
    assert err <= 1e-5, err


def test_config5_shape_finite_differences_and_f32():
    """512 x 1024 increments, width 5, depth 6, loss <W, sig> with W ~ N(0,1):
    the float64 adjoint against central differences on 64 sampled coordinates,
    and the float32-compensated adjoint against the float64 one."""
    n, L, w, d = 512, 1024, 5, 6
    rng = np.random.default_rng(4)
    inc64 = torch.from_numpy(rng.normal(0, np.sqrt(1.0 / L), size=(n * L, w))).cuda()
    off = np.arange(n + 1, dtype=np.int64) * L
    T = S.tensor_size(w, d)
    W = torch.from_numpy(rng.normal(size=(T,))).cuda()
    plan64 = S.SignaturePlan(off, w, d, "f64")
    x = inc64.clone().requires_grad_(True)
    sig = S.signature_with_grad(x, plan64)
    (sig * W).sum().backward()
    g64 = x.grad.clone()
    # central differences on sampled coordinates (one stream's signature changes)
    h = 1e-6
    picks = rng.choice(n * L * w, size=64, replace=False)
    for flat in picks:
        r, c = divmod(int(flat), w)
        s = r // L
        sub_off = np.array([0, L], dtype=np.int64)
        sub = S.SignaturePlan(sub_off, w, d, "f64")
        xs = inc64[s * L:(s + 1) * L].clone()
        xs[r - s * L, c] += h
        lp = float((sub.run(xs) * W).sum())
        xs[r - s * L, c] -= 2 * h
        lm = float((sub.run(xs) * W).sum())
        fd = (lp - lm) / (2 * h)
        assert abs(float(g64[r, c]) - fd) <= 1e-6 * max(1.0, abs(fd)), (r, c, fd, float(g64[r, c]))
    # float32 compensated mode against the float64 gradient on a 64-stream slice
    m = 64
    sl = slice(0, m * L)
    plan32 = S.SignaturePlan(off[:m + 1], w, d, "f32c")
    x32 = inc64[sl].float().clone().requires_grad_(True)
    sig32 = S.signature_with_grad(x32, plan32)
    (sig32.double() * W).sum().backward()
    planb = S.SignaturePlan(off[:m + 1], w, d, "f64")
    xb = inc64[sl].float().double().clone().requires_grad_(True)
    (S.signature_with_grad(xb, planb) * W).sum().backward()
    err = float((x32.grad.double() - xb.grad).abs().max()) / float(xb.grad.abs().max())
    assert err <= 1e-5, err


def test_shared_gradient_row_and_checkpoint_interval_invariance():
    rng = np.random.default_rng(8)
    w, d = 3, 3
    off = S.offsets_from_lengths([40, 17, 64])
    inc = torch.from_numpy(rng.normal(0, 0.3, size=(int(off[-1]), w))).cuda()
    plan = S.SignaturePlan(off, w, d, "f64")
    grads = []
    for K in (1, 5, 64, 1000):
        x = inc.clone().requires_grad_(True)
        S.signature_with_grad(x, plan, checkpoint_every=K).sum().backward()
        grads.append(x.grad)
    for g in grads[1:]:
        assert float((g - grads[0]).abs().max()) <= 1e-12 * float(grads[0].abs().max())


@pytest.mark.parametrize("w,d", [(3, 4), (5, 3), (2, 6)])
def test_adjoint_matches_forward_mode_sig_derivative(w, d):
    """<W, J v> from the forward-mode derivative (rpyb_sig_derivative, the
    reference's sig_derivative) equals <J^T W, v> from the adjoint kernel,
    for one-step streams (where the reference's recurrence is the Jacobian)."""
    from roughpy_b200 import compute as rpc
    from roughpy_b200.streams import sig_derivative_batch
    rng = np.random.default_rng(w * 7 + d)
    n = 6
    L = rpc.LieBasis(w, d).size()
    T = S.tensor_size(w, d)
    x = rng.normal(0, 0.5, (n, w))
    v = rng.normal(0, 1.0, (n, w))
    W = torch.from_numpy(rng.normal(size=(n, T))).cuda()
    lg = np.zeros((n, L))
    pt = np.zeros((n, L))
    lg[:, :w] = x
    pt[:, :w] = v
    jv = sig_derivative_batch(lg, pt, np.arange(n + 1), w, d)          # [n, T]
    fwd = (W * jv).sum(dim=1)
    plan = S.SignaturePlan(np.arange(n + 1), w, d, "f64")
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    (S.signature_with_grad(xt, plan) * W).sum().backward()
    rev = (xt.grad * torch.from_numpy(v).cuda()).sum(dim=1)
    assert float((fwd - rev).abs().max()) <= 1e-12 * max(1.0, float(fwd.abs().max()))


def _backward_call(plan, x, G, max_len, K=8):
    from roughpy_b200 import _lib
    ws_bytes = int(_lib.lib.rpyb_signature_backward_workspace_size(
        plan.code, plan.width, plan.depth, plan.n_streams, max(plan.max_len, max_len), K))
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
    gi = torch.full_like(x, 7.0)
    rc = _lib.lib.rpyb_signature_backward(
        plan.code, plan.width, plan.depth, plan.n_streams, plan.offsets.data_ptr(), max_len,
        x.data_ptr(), G.data_ptr(), G.stride(0), gi.data_ptr(), K, ws.data_ptr(), ws.numel(),
        torch.cuda.current_stream().cuda_stream)
    return rc, gi


def test_backward_rejects_streams_longer_than_max_len_and_accepts_auto():
    """The C ABI checks the caller's max_len against the offsets before any
    launch: a bound below the longest stream returns RPYB_E_INVALID and leaves
    the gradient untouched; max_len = -1 takes the longest stream."""
    from roughpy_b200 import _lib
    rng = np.random.default_rng(21)
    w, d = 3, 4
    lens = [5, 40, 17]
    off = S.offsets_from_lengths(lens)
    plan = S.SignaturePlan(off, w, d, "f64")
    x = torch.from_numpy(rng.normal(0, 0.3, size=(int(off[-1]), w))).cuda()
    G = torch.from_numpy(rng.normal(size=(len(lens), plan.size))).cuda()
    rc, gi = _backward_call(plan, x, G, max_len=39)
    torch.cuda.synchronize()
    assert rc == _lib.E_INVALID
    assert "more than max_len" in _lib.last_error()
    assert bool((gi == 7.0).all())
    rc_exact, g_exact = _backward_call(plan, x, G, max_len=40)
    rc_auto, g_auto = _backward_call(plan, x, G, max_len=-1)
    torch.cuda.synchronize()
    assert rc_exact == 0 and rc_auto == 0
    assert torch.equal(g_exact, g_auto)
    assert bool(torch.isfinite(g_auto).all())
