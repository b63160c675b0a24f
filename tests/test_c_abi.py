"""The C-ABI library loads on a CPU-only host and exports its declared API.

No kernel is launched here: only argument validation and host-side
functions (sizes, Hall basis, Lie maps) are exercised.
"""
import ctypes
import pathlib
import re

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "rpyb.h").read_text()
    return sorted(set(re.findall(r"RPYB_API\s+[\w\s\*]+?\b(rpyb_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from roughpy_b200 import _lib
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(_lib.lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_sizes():
    from roughpy_b200 import _lib
    assert "sm_100a" in _lib.version()
    assert _lib.lib.rpyb_tensor_size(4, 5) == 1365
    assert _lib.lib.rpyb_tensor_size(8, 5) == 37449
    assert _lib.lib.rpyb_tensor_size(2, 12) == 8191
    assert _lib.lib.rpyb_tensor_size(8, 6) == 299593
    assert _lib.lib.rpyb_tensor_size(0, 3) == -1


@pytest.mark.parametrize("call", [
    # bad dtype
    lambda L: L.rpyb_ft_fma(7, 2, 2, 1, 1, 1, 1, 7, 7, 7, None, None),
    # null pointers
    lambda L: L.rpyb_ft_fma(1, 2, 2, 1, None, None, None, 7, 7, 7, None, None),
    # min degree above max degree
    lambda L: L.rpyb_ft_fma(1, 2, 2, 1, 8, 8, 8, 7, 7, 7,
                            (ctypes.c_int32 * 6)(2, 1, 0, -1, 0, -1), None),
    # row stride smaller than the tensor
    lambda L: L.rpyb_ft_fma(1, 2, 2, 4, 8, 8, 8, 3, 7, 7, None, None),
    # depth out of range
    lambda L: L.rpyb_ft_exp(1, 2, 99, 1, 8, 8, 7, 7, -1, None, 0, None),
    lambda L: L.rpyb_signature(5, 2, 2, 1, 8, 8, 8, 7, None, None, 0, None),
    # dyadic tree: null handle, bad mode, row length, support
    lambda L: L.rpyb_dyadic_build(1, 3, 3, 2, 0.0, 1.0, 0, None, None, 3, None, None),
    lambda L: L.rpyb_dyadic_build(9, 3, 3, 2, 0.0, 1.0, 0, None, None, 3,
                                  ctypes.byref(ctypes.c_void_p()), None),
    lambda L: L.rpyb_dyadic_build(1, 3, 3, 2, 0.0, 1.0, 0, None, None, 5,
                                  ctypes.byref(ctypes.c_void_p()), None),
    lambda L: L.rpyb_dyadic_build(1, 3, 3, 2, 1.0, 0.0, 0, None, None, 3,
                                  ctypes.byref(ctypes.c_void_p()), None),
    lambda L: L.rpyb_dyadic_query(None, 1, None, None, 0, None, 0, None, 0, None),
    # piecewise query: bad shape, null intervals
    lambda L: L.rpyb_piecewise_query(0, 3, 0, None, None, None, 0, 0.0, 1.0, 0, 1, None, None,
                                     0, None, 0, None, 0, None),
    lambda L: L.rpyb_piecewise_query(3, 3, 0, None, None, None, 0, 0.0, 1.0, 0, 1, None, None,
                                     0, None, 0, None, 0, None),
    # signature derivative: bad dtype, offsets not starting at 0
    lambda L: L.rpyb_sig_derivative(3, 3, 3, 1, None, None, None, 6, None, 40, None, 0, None),
    lambda L: L.rpyb_sig_derivative(1, 3, 3, 1, (ctypes.c_int64 * 2)(1, 2), None, None, 14, 8,
                                    40, None, 0, None),
    # sparse map: bad dtype, negative size, null CSR, row stride below the size
    lambda L: L.rpyb_sparse_map(7, 4, 4, 1, 8, 8, 8, 8, 8, 4, 4, 1.0, None),
    lambda L: L.rpyb_sparse_map(1, -1, 4, 1, 8, 8, 8, 8, 8, 4, 4, 1.0, None),
    lambda L: L.rpyb_sparse_map(1, 4, 4, 2, None, None, None, 8, 8, 4, 4, 1.0, None),
    lambda L: L.rpyb_sparse_map(1, 4, 4, 2, 8, 8, 8, 8, 8, 3, 4, 1.0, None),
    # tensor <-> Lie maps at (3,3) (L = 14, T = 40): bad dtype, negative batch,
    # null rows, strides below the sizes
    lambda L: L.rpyb_tensor_to_lie(7, 3, 3, 1, 8, 14, 8, 40, None),
    lambda L: L.rpyb_tensor_to_lie(1, 3, 3, -1, 8, 14, 8, 40, None),
    lambda L: L.rpyb_tensor_to_lie(1, 3, 3, 2, None, 14, 8, 40, None),
    lambda L: L.rpyb_tensor_to_lie(1, 3, 3, 2, 8, 13, 8, 40, None),
    lambda L: L.rpyb_lie_to_tensor(1, 3, 3, 2, 8, 39, 8, 14, None),
])
def test_invalid_arguments_are_rejected_before_any_launch(call):
    from roughpy_b200 import _lib
    rc = call(_lib.lib)
    assert rc == _lib.E_INVALID
    assert _lib.last_error()


def test_zero_batch_is_a_no_op():
    from roughpy_b200 import _lib
    assert _lib.lib.rpyb_ft_fma(1, 2, 2, 0, None, None, None, 7, 7, 7, None, None) == 0
    assert _lib.lib.rpyb_signature(1, 2, 2, 0, None, None, None, 7, None, None, 0, None) == 0
    assert _lib.lib.rpyb_sig_derivative(1, 3, 3, 0, None, None, None, 14, None, 40, None, 0,
                                        None) == 0
    assert _lib.lib.rpyb_sparse_map(1, 4, 4, 0, None, None, None, None, None, 4, 4, 1.0,
                                    None) == 0
    assert _lib.lib.rpyb_tensor_to_lie(1, 3, 3, 0, None, 14, None, 40, None) == 0
    assert _lib.lib.rpyb_dyadic_free(None) == 0
    assert _lib.lib.rpyb_release_cached_memory() == 0


def test_python_errors_match_reference_types():
    from roughpy_b200 import _internals
    with pytest.raises(ValueError):
        _internals._basis_wd(None)
    with pytest.raises(TypeError):
        _internals._dtype_code(np.int32)


def test_noalloc_size_checks_cannot_overflow():
    """rpyb_ft_exp_noalloc bounds the batch by division, so a batch whose
    byte count would overflow int64 is rejected like any oversized one, and
    a negative batch has its own message; both before any device work."""
    from roughpy_b200 import _lib
    big = 1 << 62
    assert _lib.lib.rpyb_ft_exp_noalloc(_lib.F64, 8, 5, big, 16, 16, 37449, 37449, -1,
                                        None) == _lib.E_INVALID
    assert "static scratch" in _lib.last_error()
    assert _lib.lib.rpyb_ft_exp_noalloc(_lib.F32, 8, 5, -1, 16, 16, 37449, 37449, -1,
                                        None) == _lib.E_INVALID
    assert "negative batch" in _lib.last_error()
