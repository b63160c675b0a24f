"""CPU oracle for the B200 tensor-algebra library -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only to check (or time) the GPU path.
Nothing in ``roughpy_b200`` imports it.

Two checkers live here:

* ``librpyb_oracle.so`` (``rpyb_oracle.c``): a float64 C restatement of the
  reference algorithms, built by ``make -C oracle port``.  Python wrappers
  below loop it over batches.
* ``ref_compute()``: the reference's own ``roughpy.compute`` extension
  compiled from the reference sources into ``oracle/_ref`` (``make -C oracle
  ref``), when that build is present.

The C restatement is pinned to the reference by the golden fixtures in
``tests/golden`` (generated by the reference build) and by the reference's
known-answer tests (tests/compute/*.py), restated in ``tests/``.
"""
from __future__ import annotations

import ctypes
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
PORT_SO = HERE / "_build" / "librpyb_oracle.so"
REF_DIR = HERE / "_ref"

_lib = None


def load():
    """Load (building first if needed) the C restatement."""
    global _lib
    if _lib is not None:
        return _lib
    if not PORT_SO.exists():
        import subprocess
        subprocess.run(["make", "-C", str(HERE), "port"], check=True, capture_output=True)
    lib = ctypes.CDLL(str(PORT_SO))
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int32)
    i = ctypes.c_int
    lib.orc_tensor_size.restype = ctypes.c_int64
    lib.orc_tensor_size.argtypes = [i, i]
    lib.orc_ft_fma.argtypes = [i, i, dp, dp, dp, ip]
    lib.orc_ft_inplace_mul.argtypes = [i, i, dp, dp, ip, ctypes.c_double]
    lib.orc_ft_exp.argtypes = [i, i, dp, dp, i]
    lib.orc_ft_fmexp.argtypes = [i, i, dp, dp, dp, i]
    lib.orc_ft_log.argtypes = [i, i, dp, dp, i, i]
    lib.orc_ft_antipode.argtypes = [i, i, dp, dp]
    lib.orc_ft_adjoint_left_mul.argtypes = [i, i, dp, dp, dp, i, i, i]
    lib.orc_signature.argtypes = [i, i, ctypes.c_int64, dp, dp]
    for f in (lib.orc_ft_fma, lib.orc_ft_inplace_mul, lib.orc_ft_exp, lib.orc_ft_fmexp,
              lib.orc_ft_log, lib.orc_ft_antipode, lib.orc_ft_adjoint_left_mul,
              lib.orc_signature):
        f.restype = None
    _lib = lib
    return lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _rows(a, size):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(-1, a.shape[-1])


def _bounds(vals):
    if vals is None:
        return None
    arr = (ctypes.c_int32 * len(vals))(*[int(v) for v in vals])
    return arr


def tensor_size(width: int, depth: int) -> int:
    return int(load().orc_tensor_size(width, depth))


def ft_fma(width, depth, out, lhs, rhs, bounds=None):
    """Return out + lhs (x) rhs (batched over leading axes), float64."""
    lib = load()
    o = _rows(out, 0).copy()
    l_ = _rows(lhs, 0)
    r_ = _rows(rhs, 0)
    b = _bounds(bounds)
    for i in range(o.shape[0]):
        lib.orc_ft_fma(width, depth, _p(o[i]), _p(l_[i]), _p(r_[i]), b)
    return o.reshape(np.shape(out))


def ft_mul(width, depth, lhs, rhs):
    return ft_fma(width, depth, np.zeros_like(np.asarray(lhs, dtype=np.float64)), lhs, rhs)


def ft_inplace_mul(width, depth, lhs, rhs, bounds=None, scale=1.0):
    lib = load()
    o = _rows(lhs, 0).copy()
    r_ = _rows(rhs, 0)
    b = _bounds(bounds)
    for i in range(o.shape[0]):
        lib.orc_ft_inplace_mul(width, depth, _p(o[i]), _p(r_[i]), b, float(scale))
    return o.reshape(np.shape(lhs))


def ft_exp(width, depth, arg, out_depth=-1):
    lib = load()
    a = _rows(arg, 0)
    o = np.zeros_like(a)
    for i in range(a.shape[0]):
        lib.orc_ft_exp(width, depth, _p(o[i]), _p(a[i]), int(out_depth))
    return o.reshape(np.shape(arg))


def ft_fmexp(width, depth, mul, expo, out_depth=-1):
    lib = load()
    m = _rows(mul, 0)
    x = _rows(expo, 0)
    o = np.zeros_like(m)
    for i in range(m.shape[0]):
        lib.orc_ft_fmexp(width, depth, _p(o[i]), _p(m[i]), _p(x[i]), int(out_depth))
    return o.reshape(np.shape(mul))


def ft_log(width, depth, arg, out_depth=-1, arg_depth=-1, out_init=None):
    lib = load()
    a = _rows(arg, 0)
    o = np.zeros_like(a) if out_init is None else _rows(out_init, 0).copy()
    for i in range(a.shape[0]):
        lib.orc_ft_log(width, depth, _p(o[i]), _p(a[i]), int(out_depth), int(arg_depth))
    return o.reshape(np.shape(arg))


def antipode(width, depth, arg):
    lib = load()
    a = _rows(arg, 0)
    o = np.zeros_like(a)
    for i in range(a.shape[0]):
        lib.orc_ft_antipode(width, depth, _p(o[i]), _p(a[i]))
    return o.reshape(np.shape(arg))


def adjoint_left_mul(width, depth, op, arg, out_depth=-1, op_depth=-1, arg_depth=-1):
    lib = load()
    p = _rows(op, 0)
    a = _rows(arg, 0)
    o = np.zeros_like(a)
    for i in range(a.shape[0]):
        lib.orc_ft_adjoint_left_mul(width, depth, _p(o[i]), _p(p[i]), _p(a[i]), int(out_depth),
                                    int(op_depth), int(arg_depth))
    return o.reshape(np.shape(arg))


def signature(width, depth, increments):
    """Chen product of exp(x_t) for one stream: increments [L, width]."""
    lib = load()
    inc = np.ascontiguousarray(increments, dtype=np.float64).reshape(-1, width)
    out = np.zeros(tensor_size(width, depth))
    lib.orc_signature(width, depth, inc.shape[0], _p(inc), _p(out))
    return out


def signatures(width, depth, increments, offsets):
    """Batch of streams in CSR form (offsets[n+1] into increments rows)."""
    n = len(offsets) - 1
    out = np.zeros((n, tensor_size(width, depth)))
    for s in range(n):
        out[s] = signature(width, depth, increments[offsets[s]:offsets[s + 1]])
    return out


def ref_compute():
    """The reference ``roughpy.compute`` built from its sources, or None."""
    so = list((REF_DIR / "roughpy" / "compute").glob("_rpy_compute_internals*.so"))
    if not so:
        return None
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    try:
        from roughpy import compute  # type: ignore
    except Exception:  # pragma: no cover - build present but unusable
        return None
    return compute
