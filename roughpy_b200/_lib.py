"""ctypes binding of ``librpyb.so`` (the C ABI declared in ``include/rpyb.h``).

The library is loaded from ``roughpy_b200/_lib/librpyb.so``; there is no
fallback implementation.  Importing this module on a machine without the
built library raises ``ImportError`` with the build command.
"""
from __future__ import annotations

import ctypes
import os
import pathlib

_HERE = pathlib.Path(__file__).resolve().parent
# RPYB_LIB_PATH selects another build of the same library (e.g. a tuning variant).
LIB_PATH = pathlib.Path(os.environ.get("RPYB_LIB_PATH", _HERE / "_lib" / "librpyb.so"))

F32 = 0
F64 = 1

OK = 0
E_INVALID = -1
E_CUDA = -2
E_NOMEM = -3
E_TIMEOUT = -4
E_UNSUPPORTED = -5

if not LIB_PATH.exists():
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python roughpy_b200/build.py`")

lib = ctypes.CDLL(str(LIB_PATH))

_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_int = ctypes.c_int
_vp = ctypes.c_void_p
_sz = ctypes.c_size_t
_dbl = ctypes.c_double
_pi32 = ctypes.POINTER(ctypes.c_int32)
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pdbl = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); kept in the order of include/rpyb.h
SIGNATURES = {
    "rpyb_last_error": (ctypes.c_char_p, []),
    "rpyb_version": (ctypes.c_char_p, []),
    "rpyb_release_cached_memory": (_int, []),
    "rpyb_scratch_pool_usage": (_int, [_vp, _vp]),
    "rpyb_tensor_size": (_i64, [_i32, _i32]),
    "rpyb_ft_fma": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _vp, _i64, _i64, _i64, _pi32, _vp]),
    "rpyb_ft_mul_gather": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp,
                                  _int, _vp]),
    "rpyb_ft_mul_gather_mixed": (_int, [_i32, _i32, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _int,
                                        _vp]),
    "rpyb_ft_inplace_mul_workspace_size": (_i64, [_int, _i32, _i32, _i64]),
    "rpyb_ft_inplace_mul": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _i64, _i64, _pi32, _vp, _sz,
                                   _vp]),
    "rpyb_ft_exp_workspace_size": (_i64, [_int, _i32, _i32, _i64]),
    "rpyb_ft_exp": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _i64, _i64, _i32, _vp, _sz, _vp]),
    "rpyb_ft_exp_noalloc_max_bytes": (_i64, []),
    "rpyb_ft_exp_noalloc": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _i64, _i64, _i32, _vp]),
    "rpyb_ft_fmexp_workspace_size": (_i64, [_int, _i32, _i32, _i64]),
    "rpyb_ft_fmexp": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _vp, _i64, _i64, _i64, _i32, _vp,
                             _sz, _vp]),
    "rpyb_ft_log_workspace_size": (_i64, [_int, _i32, _i32, _i64]),
    "rpyb_ft_log": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _i64, _i64, _i32, _i32, _vp, _sz,
                           _vp]),
    "rpyb_ft_antipode": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _i64, _i64, _vp]),
    "rpyb_ft_adjoint_left_mul": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _vp, _i64, _i64, _i64,
                                        _pi32, _vp]),
    "rpyb_signature_workspace_size": (_i64, [_int, _i32, _i32, _i64]),
    "rpyb_signature": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _vp, _i64, _vp, _vp, _sz, _vp]),
    "rpyb_signature_batched_workspace_size": (_i64, [_int, _i32, _i32, _i64, _i64, _int]),
    "rpyb_signature_batched": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _i64, _vp, _i64, _vp,
                                      _vp, _vp, _sz, _vp]),
    "rpyb_sig_plan_create": (_int, [_int, _i32, _i32, _i64, _vp, _i32, _vp, _vp]),
    "rpyb_sig_plan_run": (_int, [_vp, _vp, _vp, _i64, _vp, _vp]),
    "rpyb_sig_plan_describe": (_int, [_vp, ctypes.c_char_p, _i64]),
    "rpyb_sig_plan_free": (_int, [_vp]),
    "rpyb_signature_host_device_bytes": (_i64, [_int, _i32, _i32, _i64, _vp, _i32]),
    "rpyb_signature_host": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _vp, _i64, _i32, _vp, _sz,
                                   _vp]),
    "rpyb_signature_backward_workspace_size": (_i64, [_int, _i32, _i32, _i64, _i64, _i32]),
    "rpyb_signature_backward": (_int, [_int, _i32, _i32, _i64, _vp, _i64, _vp, _vp, _i64, _vp,
                                       _i32, _vp, _sz, _vp]),
    "rpyb_lie_basis_size": (_i64, [_i32, _i32]),
    "rpyb_lie_basis_data": (_int, [_i32, _i32, _pi64, _pi64]),
    "rpyb_lie_map_csr": (_i64, [_i32, _i32, _int, _pi64, _pi64, _pdbl]),
    "rpyb_sparse_map": (_int, [_int, _i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _dbl,
                               _vp]),
    "rpyb_tensor_to_lie": (_int, [_int, _i32, _i32, _i64, _vp, _i64, _vp, _i64, _vp]),
    "rpyb_lie_to_tensor": (_int, [_int, _i32, _i32, _i64, _vp, _i64, _vp, _i64, _vp]),
    "rpyb_dyadic_dissect": (_i64, [_dbl, _dbl, _i32, _int, _vp, _vp, _i64]),
    "rpyb_dyadic_dissect_batch": (_int, [_i64, _vp, _vp, _vp, _int, _vp, _vp, _i64, _vp]),
    "rpyb_dyadic_build": (_int, [_int, _i32, _i32, _i32, _dbl, _dbl, _i64, _vp, _vp, _i32, _vp,
                                 _vp]),
    "rpyb_dyadic_save_size": (_i64, [_vp]),
    "rpyb_dyadic_save": (_i64, [_vp, _vp, _i64, _vp]),
    "rpyb_dyadic_load": (_int, [_vp, _i64, _vp, _vp]),
    "rpyb_dyadic_free": (_int, [_vp]),
    "rpyb_dyadic_range_table": (_int, [_vp, _i32, _vp]),
    "rpyb_dyadic_tree_info": (_int, [_vp, _vp, _vp, _vp]),
    "rpyb_dyadic_node_row": (_i64, [_vp, _i32, _i64]),
    "rpyb_dyadic_query": (_int, [_vp, _i64, _vp, _vp, _i32, _vp, _i64, _vp, _i64, _vp]),
    "rpyb_piecewise_query": (_int, [_i32, _i32, _i64, _vp, _vp, _vp, _i64, _dbl, _dbl, _i32,
                                    _i64, _vp, _vp, _i32, _vp, _i64, _vp, _i64, _vp]),
    "rpyb_cbh": (_int, [_i32, _i32, _i64, _vp, _vp, _i64, _vp, _i64, _vp]),
    "rpyb_sig_derivative_workspace_size": (_i64, [_int, _i32, _i32, _i64, _i64]),
    "rpyb_sig_derivative": (_int, [_int, _i32, _i32, _i64, _vp, _vp, _vp, _i64, _vp, _i64, _vp,
                                   _sz, _vp]),
}

# rpyb_sig_plan_create flag: time the schedule candidates when no cached choice exists
SIG_PLAN_TUNE = 1

# rpyb_dyadic_query: choose the dissection resolution per query as the reference does
QUERY_RESOLUTION_AUTO = -2147483648

for _name, (_res, _args) in SIGNATURES.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


class RPYBError(RuntimeError):
    """A librpyb call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[rpyb {code}] {message}")
        self.code = code


def last_error() -> str:
    msg = lib.rpyb_last_error()
    return msg.decode() if msg else ""


def check(rc: int) -> None:
    """Raise the Python exception matching a librpyb status code."""
    if rc == OK:
        return
    msg = last_error()
    if rc == E_INVALID:
        raise ValueError(msg)
    if rc == E_UNSUPPORTED:
        raise NotImplementedError(msg)
    if rc == E_NOMEM:
        raise MemoryError(msg)
    raise RPYBError(rc, msg)


def bounds(*vals) -> ctypes.Array:
    return (ctypes.c_int32 * len(vals))(*[int(v) for v in vals])


def version() -> str:
    return lib.rpyb_version().decode()
