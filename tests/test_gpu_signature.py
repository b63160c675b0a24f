"""GPU parity of the batched signature kernel.

float64 mode against the reference's fmexp-chain signatures (golden) and the
oracle at <= 1e-12; float32 compensated mode against float64 at <= 1e-6
(the accuracy bar for the compensated path), including long streams.
"""
import numpy as np
import pytest
import torch

import oracle
from roughpy_b200 import signatures as S
from tests._util import level_rel_err

pytestmark = pytest.mark.gpu


def test_f64_matches_reference_golden(golden):
    g = golden["signatures"]
    for key in g.files:
        if not key.endswith("_sig"):
            continue
        t = key[:-4]
        w, d = int(t[1:t.index("d")]), int(t[t.index("d") + 1:])
        got = S.signature(g[f"{t}_inc"], g[f"{t}_offsets"], depth=d, mode="f64")
        assert level_rel_err(got, g[key], w, d) <= 1e-12, t


@pytest.mark.parametrize("w,d", [(2, 2), (2, 7), (3, 5), (4, 5), (5, 6), (6, 5), (7, 3),
                                 (8, 5), (2, 9), (9, 2), (3, 1), (4, 0), (10, 3)])
def test_f64_against_oracle_uneven(w, d):
    rng = np.random.default_rng(w * 31 + d)
    lens = rng.integers(0, 40, size=9)
    lens[0] = 0
    off = S.offsets_from_lengths(lens)
    inc = rng.normal(0, 0.3, size=(int(off[-1]), w))
    got = S.signature(inc, off, depth=d, mode="f64")
    want = oracle.signatures(w, d, inc, off)
    assert level_rel_err(got, want, w, d) <= 1e-12


@pytest.mark.parametrize("w,d,maxlen", [(8, 5, 4096), (4, 5, 1024), (5, 6, 1024), (6, 5, 2048)])
def test_f32c_within_1e6_of_f64(w, d, maxlen):
    rng = np.random.default_rng(2)
    n = 24
    lens = rng.integers(16, maxlen + 1, size=n)
    off = S.offsets_from_lengths(lens)
    inc = np.concatenate([rng.normal(0, np.sqrt(1.0 / L), size=(L, w)) for L in lens])
    inc32 = inc.astype(np.float32)
    ref = S.signature(inc32.astype(np.float64), off, depth=d, mode="f64")
    got = S.signature(inc32, off, depth=d, mode="f32c")
    assert got.dtype == np.float32
    err = level_rel_err(got, ref, w, d)
    assert err <= 1e-6, err


def test_f64_gpu_equals_oracle_on_config1_sample():
    rng = np.random.default_rng(0)
    n, L, w, d = 16, 128, 4, 5
    inc = rng.normal(0, np.sqrt(1 / 128), size=(n * L, w))
    off = np.arange(n + 1, dtype=np.int64) * L
    got = S.signature(inc, off, depth=d, mode="f64")
    want = oracle.signatures(w, d, inc, off)
    assert level_rel_err(got, want, w, d) <= 1e-12


def test_plan_reuse_and_torch_inputs():
    rng = np.random.default_rng(9)
    w, d = 8, 5
    lens = np.array([5, 300, 17, 0, 64])
    off = S.offsets_from_lengths(lens)
    inc = torch.from_numpy(rng.normal(0, 0.05, size=(int(off[-1]), w)).astype(np.float32)).cuda()
    plan = S.SignaturePlan(off, w, d, "f32c")
    a = plan.run(inc).clone()
    b = plan.run(inc)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert float(a[3, 0]) == 1.0 and float(a[3, 1:].abs().max()) == 0.0


@pytest.mark.parametrize("mode,chunks", [("f32c", 1), ("f32c", 5), ("f64", 3)])
def test_host_pipelined_entry_matches_device_path(mode, chunks):
    rng = np.random.default_rng(13)
    w, d = 8, 5
    lens = rng.integers(0, 300, size=37)
    off = S.offsets_from_lengths(lens)
    dt = np.float64 if mode == "f64" else np.float32
    inc = rng.normal(0, 0.05, size=(int(off[-1]), w)).astype(dt)
    plan = S.SignaturePlan(off, w, d, mode)
    want = plan.run(torch.from_numpy(inc).cuda()).cpu()
    inc_h = torch.from_numpy(inc).pin_memory()
    out_h = torch.full((len(lens), plan.size), float("nan"), dtype=plan.dtype).pin_memory()
    plan.run_host_pipelined(inc_h, out_h, n_chunks=chunks)
    torch.cuda.synchronize()
    if plan.schedule()["seg"] == 0:
        assert torch.equal(out_h, want)
    else:
        # the host entry runs whole streams; a tuned plan may cut them into
        # time segments: equal up to the mode's rounding
        tol = 1e-12 if mode == "f64" else 2e-6
        o, g = out_h.numpy(), want.numpy()
        assert max(level_rel_err(o[s:s + 1], g[s:s + 1], w, d) for s in range(len(lens))) <= tol


@pytest.mark.parametrize("mode", ["f64", "f32c"])
def test_plan_cuda_graph_replays_with_refilled_inputs(mode):
    """SignaturePlan.capture: the captured launch, replayed after refilling
    the static increments in place, gives exactly the direct launch's result
    on the new increments; two replays in a row."""
    rng = np.random.default_rng(8)
    w, d = 4, 5
    lens = rng.integers(0, 300, size=40)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    plan = S.SignaturePlan(off, w, d, mode)
    x = torch.from_numpy(rng.normal(0, 0.1, size=(int(off[-1]), w))).to("cuda", plan.dtype)
    graph, gout = plan.capture(x)
    for trial in range(2):
        new = torch.from_numpy(rng.normal(0, 0.1, size=(int(off[-1]), w))).to("cuda", plan.dtype)
        x.copy_(new)
        graph.replay()
        want = plan.run(new)
        torch.cuda.synchronize()
        assert torch.equal(gout, want), trial


@pytest.mark.parametrize("w,d", [(8, 5), (4, 5), (3, 7)])
def test_report_error_matches_the_float64_comparison(w, d):
    """SignaturePlan.run(report_error=True): the per-stream error equals the
    per-level relative error of the float32 result against the float64 path
    on the same increments, to 1e-12; rpyb_signature_batched reports the same."""
    from roughpy_b200 import _lib
    rng = np.random.default_rng(31 + w)
    lens = rng.integers(0, 700, size=19)
    lens[3] = 0
    off = S.offsets_from_lengths(lens)
    inc = (rng.normal(size=(int(off[-1]), w)) / 20.0).astype(np.float32)
    plan = S.SignaturePlan(off, w, d, "f32c")
    x = torch.from_numpy(inc).cuda()
    out, err = plan.run(x, report_error=True)
    plain = plan.run(x)
    ref = S.SignaturePlan(off, w, d, "f64").run(x.double())
    torch.cuda.synchronize()
    assert torch.equal(out, plain)
    got = err.cpu().numpy()
    o, r = out.cpu().numpy(), ref.cpu().numpy()
    want = np.array([level_rel_err(o[s:s + 1], r[s:s + 1], w, d) for s in range(len(lens))])
    assert np.max(np.abs(got - want)) <= 1e-12
    assert got[3] == 0.0 and np.max(got) <= 1e-6
    # the stateless entry point
    nb = int(_lib.lib.rpyb_signature_batched_workspace_size(_lib.F32, w, d, len(lens),
                                                             int(off[-1]), 1))
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    out2 = torch.empty_like(out)
    err2 = torch.empty_like(err)
    _lib.check(_lib.lib.rpyb_signature_batched(
        _lib.F32, w, d, len(lens), plan.offsets.data_ptr(), x.data_ptr(), int(off[-1]),
        out2.data_ptr(), plan.size, plan.order.data_ptr(), err2.data_ptr(), ws.data_ptr(),
        nb, torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    if plan.schedule()["seg"] == 0:
        # whole streams: the same arithmetic whatever the lane shape
        assert torch.equal(out2, out) and torch.equal(err2, err)
    else:
        # the tuned plan cuts streams into time segments merged by Chen
        # products: the same values up to float32 rounding
        o2 = out2.cpu().numpy()
        assert max(level_rel_err(o2[s:s + 1], o[s:s + 1], w, d) for s in range(len(lens))) <= 2e-6
        assert float((err2 - err).abs().max()) <= 1e-6
    _, e64 = S.SignaturePlan(off, w, d, "f64").run(x.double(), report_error=True)
    assert float(e64.abs().max()) == 0.0
