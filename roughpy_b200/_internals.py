"""Drop-in for RoughPy's ``roughpy.compute._rpy_compute_internals`` extension.

Same function names, argument names and defaults as the reference method
table (roughpy/compute/_src/roughpy_compute_module.c:12-59): ``dense_ft_fma``,
``dense_ft_inplace_mul``, ``dense_ft_antipode``, ``dense_ft_exp``,
``dense_ft_fmexp``, ``dense_ft_log``, ``dense_ft_adjoint_left_mul``,
``dense_lie_to_tensor``, ``dense_tensor_to_lie`` plus the ``TensorBasis`` and
``LieBasis`` types.  Every call runs on the GPU through ``librpyb.so``.

Arrays may be NumPy arrays (copied to the device and the results copied back
into the caller's ``out`` array, as the reference writes in place) or CUDA
``torch.Tensor`` objects (used in place, no copies).  Leading dimensions are
batch dimensions and must match between arguments; the last axis holds the
tensor (roughpy/compute/_src/py_ternary_array_fn.hpp:70-161).  Errors follow
the reference: ``TypeError`` for dtype problems, ``ValueError`` for shapes
and degree bounds.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

__all__ = [
    "TensorBasis", "LieBasis", "SparseMatrix", "dense_ft_fma", "dense_ft_inplace_mul",
    "dense_ft_antipode", "dense_ft_exp", "dense_ft_fmexp", "dense_ft_log",
    "dense_ft_adjoint_left_mul", "dense_lie_to_tensor", "dense_tensor_to_lie",
    "check_lie_basis_data",
]


# --------------------------------------------------------------------- bases
def _standard_degree_begin(width: int, depth: int) -> np.ndarray:
    db = np.zeros(depth + 2, dtype=np.intp)
    for i in range(1, depth + 2):
        db[i] = 1 + width * db[i - 1]
    return db


class TensorBasis:
    """Dense tensor basis metadata (roughpy/compute/_src/tensor_basis.c)."""

    def __init__(self, width: int, depth: int):
        width = int(width)
        depth = int(depth)
        if width < 1 or depth < 0:
            raise ValueError("width must be >= 1 and depth >= 0")
        self.width = width
        self.depth = depth
        self.degree_begin = _standard_degree_begin(width, depth)

    def size(self) -> int:
        return int(self.degree_begin[self.depth + 1])

    def truncate(self, depth: int) -> "TensorBasis":
        return TensorBasis(self.width, min(self.depth, int(depth)))

    def __eq__(self, other):
        return (isinstance(other, TensorBasis) and other.width == self.width
                and other.depth == self.depth)

    def __hash__(self):
        return hash(("TensorBasis", self.width, self.depth))

    def __repr__(self):
        return f"TensorBasis({self.width}, {self.depth})"


class SparseMatrix:
    """CSR matrix with float64 (or cast) values; ``rows x cols``."""

    def __init__(self, indptr, indices, data, shape):
        self.indptr = np.asarray(indptr, dtype=np.int64)
        self.indices = np.asarray(indices, dtype=np.int64)
        self.data = np.asarray(data)
        self.shape = tuple(int(s) for s in shape)
        self._dev = {}

    @property
    def nnz(self) -> int:
        return int(self.indices.shape[0])

    def todense(self) -> np.ndarray:
        out = np.zeros(self.shape, dtype=self.data.dtype)
        for r in range(self.shape[0]):
            s, e = self.indptr[r], self.indptr[r + 1]
            out[r, self.indices[s:e]] += self.data[s:e]
        return out

    def device_arrays(self, device):
        key = str(device)
        if key not in self._dev:
            self._dev[key] = (
                torch.from_numpy(self.indptr).to(device),
                torch.from_numpy(self.indices).to(device),
                torch.from_numpy(np.ascontiguousarray(self.data, dtype=np.float64)).to(device),
            )
        return self._dev[key]


class LieBasis:
    """Hall basis with RoughPy's greedy construction.

    ``data`` is an ``(n + 1, 2)`` intp array of parent pairs with a null row
    0, ``degree_begin`` has ``depth + 2`` entries; both are produced by the
    C++ builder in ``librpyb.so`` (same rule as
    roughpy/compute/_src/lie_basis.c:201-337).
    """

    def __init__(self, width: int, depth: int):
        self.width = int(width)
        self.depth = int(depth)
        n = int(_lib.lib.rpyb_lie_basis_size(self.width, self.depth))
        if n < 0:
            raise ValueError(_lib.last_error())
        data = np.zeros((n + 1, 2), dtype=np.int64)
        db = np.zeros(self.depth + 2, dtype=np.int64)
        _lib.check(_lib.lib.rpyb_lie_basis_data(
            self.width, self.depth,
            data.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            db.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        self.data = data.astype(np.intp)
        self.degree_begin = db.astype(np.intp)
        self._maps = {}

    def size(self) -> int:
        return int(self.degree_begin[self.depth + 1]) - 1

    # Value semantics as in the reference type (roughpy/compute/_src/
    # lie_basis.c:520-610): bases are equal when width, depth, degree_begin
    # and the Hall data agree, and the hash covers the same fields.
    def _key(self):
        n = self.size() + 1
        return (self.width, self.depth, self.degree_begin[:self.depth + 2].tobytes(),
                self.data[:n].tobytes())

    def __hash__(self):
        h = self.__dict__.get("_hash")
        if h is None:
            h = hash(("LieBasis",) + self._key())
            self._hash = h
        return h

    def __eq__(self, other):
        if not isinstance(other, LieBasis):
            return NotImplemented
        return self._key() == other._key()

    def __ne__(self, other):
        eq = self.__eq__(other)
        return eq if eq is NotImplemented else not eq

    def _csr(self, which: int, dtype) -> SparseMatrix:
        key = (which, np.dtype(dtype).str)
        if key not in self._maps:
            nnz = int(_lib.lib.rpyb_lie_map_csr(self.width, self.depth, which, None, None, None))
            if nnz < 0:
                _lib.check(nnz)
            tsize = TensorBasis(self.width, self.depth).size()
            rows = tsize if which == 0 else self.size()
            cols = self.size() if which == 0 else tsize
            ptr = np.zeros(rows + 1, dtype=np.int64)
            idx = np.zeros(nnz, dtype=np.int64)
            val = np.zeros(nnz, dtype=np.float64)
            _lib.lib.rpyb_lie_map_csr(
                self.width, self.depth, which,
                ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                val.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            self._maps[key] = SparseMatrix(ptr, idx, val.astype(dtype), (rows, cols))
        return self._maps[key]

    def get_l2t_matrix(self, dtype=np.float64) -> SparseMatrix:
        """Lie -> tensor map, ``tensor_size x lie_size`` (lie_basis.c:902-973)."""
        return self._csr(0, dtype)

    def get_t2l_matrix(self, dtype=np.float64) -> SparseMatrix:
        """Tensor -> Lie map (Dynkin r-bracketing / degree), ``lie_size x tensor_size``."""
        return self._csr(1, dtype)

    def __repr__(self):
        return f"LieBasis({self.width}, {self.depth})"


def check_lie_basis_data(width, depth, data, degree_begin=None) -> bool:
    """True when ``data`` equals the greedy Hall set for (width, depth)."""
    ref = LieBasis(width, depth)
    data = np.asarray(data)
    return data.shape == ref.data.shape and bool(np.all(data == ref.data))


# -------------------------------------------------------------- array glue
def _dtype_code(dt) -> int:
    if dt in (np.float64, torch.float64):
        return _lib.F64
    if dt in (np.float32, torch.float32):
        return _lib.F32
    raise TypeError("unsupported dtype")


def _basis_wd(basis):
    if basis is None:
        raise ValueError("basis object is null")
    w = int(basis.width)
    d = int(basis.depth)
    db = getattr(basis, "degree_begin", None)
    if db is not None:
        db = np.asarray(db)
        if db.ndim != 1 or db.shape[0] < d + 2:
            raise ValueError("degree_begin must have at least depth + 2 elements")
        if not np.array_equal(db[:d + 2], _standard_degree_begin(w, d)):
            raise NotImplementedError("only the standard dense degree layout is supported")
    return w, d


class _Arg:
    """One array argument: a CUDA tensor view of shape (batch, n) plus writeback."""

    def __init__(self, obj, name: str, need: int, writable: bool, device=None):
        self.name = name
        self.obj = obj
        self.is_numpy = isinstance(obj, np.ndarray)
        if self.is_numpy:
            if obj.dtype not in (np.float32, np.float64):
                raise TypeError(f"{name}: unsupported dtype")
            host = np.ascontiguousarray(obj)
            t = torch.from_numpy(host)
            self.t = t.to(device or "cuda", non_blocking=False)
        elif isinstance(obj, torch.Tensor):
            if obj.dtype not in (torch.float32, torch.float64):
                raise TypeError(f"{name}: unsupported dtype")
            if not obj.is_cuda:
                self.t = obj.contiguous().to(device or "cuda")
            else:
                self.t = obj if obj.is_contiguous() else obj.contiguous()
        else:
            raise TypeError(f"{name} must be a numpy array or a torch tensor")
        if self.t.dim() < 1:
            raise ValueError("invalid shape")
        self.lead = tuple(self.t.shape[:-1])
        self.n = int(self.t.shape[-1])
        if self.n < need:
            raise ValueError(f"{name}: last axis has {self.n} entries, needs {need}")
        self.rows = self.t.reshape(-1, self.n)
        self.writable = writable

    @property
    def dtype_code(self):
        return _dtype_code(self.t.dtype)

    @property
    def batch(self) -> int:
        return int(self.rows.shape[0])

    def ptr(self) -> int:
        return self.rows.data_ptr()

    def finish(self):
        if not self.writable:
            return
        if self.is_numpy:
            np.copyto(self.obj, self.rows.reshape(self.obj.shape).cpu().numpy())
        elif isinstance(self.obj, torch.Tensor) and self.rows.data_ptr() != self.obj.data_ptr():
            self.obj.copy_(self.rows.reshape(self.obj.shape))


def _stream_ptr(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _check_same(out: _Arg, *others: _Arg):
    for o in others:
        if o.t.dtype != out.t.dtype:
            raise TypeError(f"{o.name} must have the same dtype as out")
        if o.lead != out.lead:
            raise ValueError(f"{o.name} and out must have the same shape")


def _workspace(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


# ------------------------------------------------------------- free tensors
def dense_ft_fma(out, lhs, rhs, basis, out_depth=-1, lhs_depth=-1, rhs_depth=-1):
    """out += lhs (x) rhs (roughpy/compute/_src/dense_basic.cpp:85-151)."""
    w, d = _basis_wd(basis)
    size = int(_lib.lib.rpyb_tensor_size(w, d))
    o = _Arg(out, "out", size, True)
    lh = _Arg(lhs, "lhs", size, False, o.t.device)
    rh = _Arg(rhs, "rhs", size, False, o.t.device)
    _check_same(o, lh, rh)
    b = _lib.bounds(0, out_depth, 0, lhs_depth, 0, rhs_depth)
    _lib.check(_lib.lib.rpyb_ft_fma(o.dtype_code, w, d, o.batch, o.ptr(), lh.ptr(), rh.ptr(),
                                    o.n, lh.n, rh.n, b, _stream_ptr(o.t)))
    o.finish()


def dense_ft_inplace_mul(lhs, rhs, basis, out_depth=-1, rhs_depth=-1):
    """lhs <- lhs (x) rhs (roughpy/compute/_src/dense_basic.cpp:193-237)."""
    w, d = _basis_wd(basis)
    size = int(_lib.lib.rpyb_tensor_size(w, d))
    lh = _Arg(lhs, "lhs", size, True)
    rh = _Arg(rhs, "rhs", size, False, lh.t.device)
    _check_same(lh, rh)
    b = _lib.bounds(0, out_depth, 0, rhs_depth)
    ws = _workspace(_lib.lib.rpyb_ft_inplace_mul_workspace_size(lh.dtype_code, w, d, lh.batch),
                    lh.t.device)
    _lib.check(_lib.lib.rpyb_ft_inplace_mul(lh.dtype_code, w, d, lh.batch, lh.ptr(), rh.ptr(),
                                            lh.n, rh.n, b, ws.data_ptr(), ws.numel(),
                                            _stream_ptr(lh.t)))
    lh.finish()


def dense_ft_antipode(out, arg, basis, out_depth=-1, arg_depth=-1):
    """out <- antipode(arg) (roughpy/compute/_src/dense_basic.cpp:295-334)."""
    w, d = _basis_wd(basis)
    size = int(_lib.lib.rpyb_tensor_size(w, d))
    o = _Arg(out, "out", size, True)
    a = _Arg(arg, "arg", size, False, o.t.device)
    _check_same(o, a)
    _lib.check(_lib.lib.rpyb_ft_antipode(o.dtype_code, w, d, o.batch, o.ptr(), a.ptr(), o.n, a.n,
                                         _stream_ptr(o.t)))
    o.finish()


def dense_ft_exp(out, arg, basis, out_depth=-1, arg_depth=-1):
    """out <- exp(arg) (roughpy/compute/_src/dense_intermediate.cpp:62-96)."""
    w, d = _basis_wd(basis)
    size = int(_lib.lib.rpyb_tensor_size(w, d))
    o = _Arg(out, "out", size, True)
    a = _Arg(arg, "arg", size, False, o.t.device)
    _check_same(o, a)
    ws = _workspace(_lib.lib.rpyb_ft_exp_workspace_size(o.dtype_code, w, d, o.batch), o.t.device)
    _lib.check(_lib.lib.rpyb_ft_exp(o.dtype_code, w, d, o.batch, o.ptr(), a.ptr(), o.n, a.n,
                                    int(out_depth), ws.data_ptr(), ws.numel(), _stream_ptr(o.t)))
    o.finish()


def dense_ft_fmexp(out, multiplier, exponent, basis, out_depth=-1, multiplier_depth=-1,
                   exponent_depth=-1):
    """out <- multiplier * exp(exponent) (dense_intermediate.cpp:127-196)."""
    w, d = _basis_wd(basis)
    size = int(_lib.lib.rpyb_tensor_size(w, d))
    o = _Arg(out, "out", size, True)
    m = _Arg(multiplier, "multiplier", size, False, o.t.device)
    x = _Arg(exponent, "exponent", size, False, o.t.device)
    _check_same(o, m, x)
    ws = _workspace(_lib.lib.rpyb_ft_fmexp_workspace_size(o.dtype_code, w, d, o.batch),
                    o.t.device)
    _lib.check(_lib.lib.rpyb_ft_fmexp(o.dtype_code, w, d, o.batch, o.ptr(), m.ptr(), x.ptr(),
                                      o.n, m.n, x.n, int(out_depth), ws.data_ptr(), ws.numel(),
                                      _stream_ptr(o.t)))
    o.finish()


def dense_ft_log(out, arg, basis, out_depth=-1, arg_depth=-1):
    """out <- log(arg), float64 series (dense_intermediate.cpp:204-294)."""
    w, d = _basis_wd(basis)
    size = int(_lib.lib.rpyb_tensor_size(w, d))
    o = _Arg(out, "out", size, True)
    a = _Arg(arg, "arg", size, False, o.t.device)
    _check_same(o, a)
    ws = _workspace(_lib.lib.rpyb_ft_log_workspace_size(o.dtype_code, w, d, o.batch), o.t.device)
    _lib.check(_lib.lib.rpyb_ft_log(o.dtype_code, w, d, o.batch, o.ptr(), a.ptr(), o.n, a.n,
                                    int(out_depth), int(arg_depth), ws.data_ptr(), ws.numel(),
                                    _stream_ptr(o.t)))
    o.finish()


def dense_ft_adjoint_left_mul(out, operator, argument, basis, out_depth=-1, lhs_depth=-1,
                              rhs_depth=-1):
    """out += L*_operator(argument) (roughpy/compute/_src/dense_basic.cpp:387-440)."""
    w, d = _basis_wd(basis)
    size = int(_lib.lib.rpyb_tensor_size(w, d))
    o = _Arg(out, "out", size, True)
    op = _Arg(operator, "operator", size, False, o.t.device)
    ar = _Arg(argument, "argument", size, False, o.t.device)
    _check_same(o, op, ar)
    b = _lib.bounds(out_depth, lhs_depth, rhs_depth)
    _lib.check(_lib.lib.rpyb_ft_adjoint_left_mul(o.dtype_code, w, d, o.batch, o.ptr(), op.ptr(),
                                                 ar.ptr(), o.n, op.n, ar.n, b, _stream_ptr(o.t)))
    o.finish()


# ------------------------------------------------------------------ Lie maps
def _apply_csr(o: _Arg, a: _Arg, matrix: SparseMatrix, scale):
    ptr, idx, val = matrix.device_arrays(o.t.device)
    rows, cols = matrix.shape
    if o.n < rows or a.n < cols:
        raise ValueError("array sizes do not match the map")
    s = 1.0 if scale is None else float(scale)
    _lib.check(_lib.lib.rpyb_sparse_map(o.dtype_code, rows, cols, o.batch, ptr.data_ptr(),
                                        idx.data_ptr(), val.data_ptr(), o.ptr(), a.ptr(), o.n,
                                        a.n, s, _stream_ptr(o.t)))


def dense_lie_to_tensor(out, arg, l2t_matrix, lie_basis, tensor_basis, scale_factor=None):
    """out += scale * l2t(arg) (roughpy/compute/_src/dense_basic.cpp:564-1040)."""
    o = _Arg(out, "out", 1, True)
    a = _Arg(arg, "arg", 1, False, o.t.device)
    _check_same(o, a)
    _apply_csr(o, a, l2t_matrix, scale_factor)
    o.finish()


def dense_tensor_to_lie(out, arg, t2l_matrix, lie_basis, tensor_basis, scale_factor=None):
    """out += scale * t2l(arg) (roughpy/compute/_src/dense_basic.cpp:1055-1150)."""
    o = _Arg(out, "out", 1, True)
    a = _Arg(arg, "arg", 1, False, o.t.device)
    _check_same(o, a)
    _apply_csr(o, a, t2l_matrix, scale_factor)
    o.finish()
