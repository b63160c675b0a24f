"""rpyb_ft_exp_noalloc: the tensor exponential for callers that cannot allocate
device memory (a host application owning a fixed device pool, a thread where
an allocation would synchronise the device, a callback that forbids it).  It
takes its scratch from a static device array instead of a workspace.

This file is collected last on purpose.  Each test compares the allocation-
free entry point with the regular rpyb_ft_exp through the C ABI, on two calls
in a row (the static scratch keeps the previous call's contents), and runs the
same way alone in a fresh process or after the rest of the suite.
"""
import numpy as np
import pytest
import torch

from roughpy_b200 import _lib
from tests._util import level_rel_err

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-12, torch.float32: 2e-6}


def _exp_regular(code, w, d, x, out_depth=-1):
    out = torch.zeros_like(x)
    T = x.shape[1]
    ws_bytes = int(_lib.lib.rpyb_ft_exp_workspace_size(code, w, d, x.shape[0]))
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=x.device)
    _lib.check(_lib.lib.rpyb_ft_exp(code, w, d, x.shape[0], out.data_ptr(), x.data_ptr(), T, T,
                                    out_depth, ws.data_ptr(), ws.numel(),
                                    torch.cuda.current_stream().cuda_stream))
    return out


def _exp_noalloc(code, w, d, x, out_depth=-1):
    out = torch.zeros_like(x)
    T = x.shape[1]
    _lib.check(_lib.lib.rpyb_ft_exp_noalloc(code, w, d, x.shape[0], out.data_ptr(),
                                            x.data_ptr(), T, T, out_depth,
                                            torch.cuda.current_stream().cuda_stream))
    return out


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("w,d,batch", [(4, 5, 64), (8, 5, 4), (2, 6, 3), (3, 4, 1)])
def test_noalloc_exp_matches_regular_exp_twice(dtype, w, d, batch):
    code = _lib.F64 if dtype == torch.float64 else _lib.F32
    T = int(_lib.lib.rpyb_tensor_size(w, d))
    rng = np.random.default_rng(w * 10 + d)
    for call in range(2):
        x = torch.from_numpy(rng.normal(0, 0.5, size=(batch, T))).to("cuda", dtype)
        want = _exp_regular(code, w, d, x)
        got = _exp_noalloc(code, w, d, x)
        torch.cuda.synchronize()
        err = level_rel_err(got.cpu().numpy(), want.cpu().numpy(), w, d)
        assert err <= TOL[dtype], (call, err)


def test_noalloc_rejects_sizes_beyond_the_static_scratch():
    cap = int(_lib.lib.rpyb_ft_exp_noalloc_max_bytes())
    assert cap == 8 << 20
    w, d = 8, 5
    T = int(_lib.lib.rpyb_tensor_size(w, d))
    batch = cap // (T * 8) + 1
    rc = _lib.lib.rpyb_ft_exp_noalloc(_lib.F64, w, d, batch, 16, 16, T, T, -1, None)
    assert rc == _lib.E_INVALID
    assert "static scratch" in _lib.last_error()


def _pool_usage():
    import ctypes
    used, reserved = ctypes.c_int64(), ctypes.c_int64()
    _lib.check(_lib.lib.rpyb_scratch_pool_usage(ctypes.byref(used), ctypes.byref(reserved)))
    return used.value, reserved.value


def test_noalloc_takes_nothing_from_the_library_pool():
    """The contract itself: two calls leave the library's scratch pool empty
    (no pooled allocation in use or reserved), while the regular entry point
    given no workspace does draw on it, which shows that the probe sees a
    pooled allocation when one happens."""
    w, d, batch = 4, 5, 64
    T = int(_lib.lib.rpyb_tensor_size(w, d))
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.normal(0, 0.5, size=(batch, T))).to("cuda", torch.float64)
    torch.cuda.synchronize()
    _lib.check(_lib.lib.rpyb_release_cached_memory())
    before = _pool_usage()
    assert before == (0, 0)
    for _ in range(2):
        _exp_noalloc(_lib.F64, w, d, x)
    torch.cuda.synchronize()
    assert _pool_usage() == before
    out = torch.zeros_like(x)
    _lib.check(_lib.lib.rpyb_ft_exp(_lib.F64, w, d, batch, out.data_ptr(), x.data_ptr(), T, T, -1,
                                    None, 0, torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert _pool_usage()[1] >= batch * T * 8
    _lib.check(_lib.lib.rpyb_release_cached_memory())
