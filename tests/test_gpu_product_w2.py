"""The width-2 product kernel for float64 rows (lanes owning the last five
letters, levels >= 8 of products reaching level 10) gives the same bits as the blocked width-2 kernel it
replaces there (RPYB_W2_KERNEL=0, read once per process, so the blocked
results come from a child process), for products, FMAs and the Horner series
built on them; float32 rows keep the blocked kernel, and the same comparison
checks that the switch leaves them alone.  Both dtypes match the oracle."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHAPES = [(2, 9, 3), (2, 10, 5), (2, 12, 3)]   # depth 9: below the kernel's cutoff


def compute_all():
    """Every width-2 result the comparison covers, keyed by name."""
    from roughpy_b200 import _internals as I
    from roughpy_b200 import compute as rpc
    from tests._util import level_scaled
    res = {}
    for w, d, n in SHAPES:
        basis = rpc.TensorBasis(w, d)
        rng = np.random.default_rng(7 + d)
        A, B, C = (level_scaled(rng, w, d, n) for _ in range(3))
        X = level_scaled(rng, w, d, n)
        X[:, 0] = 0.0
        Y = level_scaled(rng, w, d, n)
        Y[:, 0] = 1.0
        for dt in (np.float64, np.float32):
            t = f"w{w}d{d}_{np.dtype(dt).name}"
            a, b, c, x, y = (v.astype(dt) for v in (A, B, C, X, Y))
            got = a.copy()
            I.dense_ft_fma(got, b, c, basis)
            res[t + "_fma"] = got
            res[t + "_mul"] = rpc.ft_mul(rpc.FreeTensor(b, basis), rpc.FreeTensor(c, basis)).data
            res[t + "_exp"] = rpc.ft_exp(rpc.FreeTensor(x, basis)).data
            res[t + "_log"] = rpc.ft_log(rpc.FreeTensor(y, basis)).data
            res[t + "_fmexp"] = rpc.ft_fmexp(rpc.FreeTensor(y, basis), rpc.FreeTensor(x, basis)).data
    return {k: np.asarray(v) for k, v in res.items()}


def test_w2_kernel_equals_blocked_kernel_bitwise(tmp_path):
    out = tmp_path / "blocked.npz"
    code = (f"import sys; sys.path.insert(0, {ROOT!r}); import numpy as np; "
            f"from tests.test_gpu_product_w2 import compute_all; "
            f"np.savez({str(out)!r}, **compute_all())")
    env = dict(os.environ, RPYB_W2_KERNEL="0")
    subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, check=True, timeout=600)
    blocked = np.load(out)
    lane = compute_all()
    assert set(blocked.files) == set(lane)
    for k in lane:
        assert lane[k].dtype == blocked[k].dtype, k
        assert np.array_equal(lane[k], blocked[k]), k


@pytest.mark.parametrize("w,d,n", SHAPES)
def test_w2_kernel_against_oracle(w, d, n):
    import oracle
    from roughpy_b200 import _internals as I
    from roughpy_b200 import compute as rpc
    from tests._util import level_rel_err, level_scaled
    rng = np.random.default_rng(40 + d)
    A, B, C = (level_scaled(rng, w, d, n) for _ in range(3))
    basis = rpc.TensorBasis(w, d)
    for dt, tol in ((np.float64, 1e-12), (np.float32, 2e-6)):
        a, b, c = (v.astype(dt) for v in (A, B, C))
        want = oracle.ft_fma(w, d, a, b, c)
        got = a.copy()
        I.dense_ft_fma(got, b, c, basis)
        assert level_rel_err(got, want, w, d) <= tol, dt
