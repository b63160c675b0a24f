"""GPU drop-in for ``roughpy.compute`` (roughpy/compute/__init__.py:129-375).

The public names, signatures and calling conventions match the reference
module, so ``from roughpy_b200 import compute as rpc`` replaces
``from roughpy import compute as rpc``.  Tensors carry their data in
``.data``: a NumPy array (results come back as NumPy, computed on the GPU)
or a CUDA ``torch.Tensor`` (computed in place, no host copies).
"""
from __future__ import annotations

import typing
from dataclasses import dataclass

import numpy as np
import torch

from . import _internals

__all__ = [
    "TensorBasis", "LieBasis", "SparseMatrix", "DenseFreeTensor", "DenseShuffleTensor",
    "DenseLie", "FreeTensor", "ShuffleTensor", "Lie", "check_lie_basis_data", "ft_fma",
    "ft_mul", "ft_inplace_mul", "antipode", "ft_exp", "ft_log", "ft_fmexp",
    "ft_adjoint_left_mul", "lie_to_tensor", "tensor_to_lie",
]

TensorBasis = _internals.TensorBasis
LieBasis = _internals.LieBasis
SparseMatrix = _internals.SparseMatrix
check_lie_basis_data = _internals.check_lie_basis_data


@dataclass()
class DenseFreeTensor:
    data: typing.Any
    basis: TensorBasis


@dataclass()
class DenseShuffleTensor:
    data: typing.Any
    basis: TensorBasis


@dataclass()
class DenseLie:
    data: typing.Any
    basis: LieBasis


FreeTensor = DenseFreeTensor
ShuffleTensor = DenseShuffleTensor
Lie = DenseLie


def _check_basis_compat(out_basis, *other_bases):
    for i, basis in enumerate(other_bases):
        if basis.width != out_basis.width:
            raise ValueError(f"Incompatible width for basis {i}")


def _zeros_like(data, n=None):
    if isinstance(data, torch.Tensor):
        shape = data.shape if n is None else (*data.shape[:-1], n)
        return torch.zeros(shape, dtype=data.dtype, device=data.device)
    shape = data.shape if n is None else (*data.shape[:-1], n)
    return np.zeros(shape, dtype=data.dtype)


def _float_dtype(data):
    dt = data.dtype
    if dt in (np.float32, np.float64, torch.float32, torch.float64):
        return dt
    raise ValueError(f"Unsupported dtype {dt}")


def ft_fma(a: FreeTensor, b: FreeTensor, c: FreeTensor, **kwargs):
    """a = b * c + a.  As in the reference, c's depth is passed as the output depth."""
    _check_basis_compat(a.basis, b.basis, c.basis)
    _internals.dense_ft_fma(a.data, b.data, c.data, b.basis, c.basis.depth)


def ft_mul(a: FreeTensor, b: FreeTensor, **kwargs) -> FreeTensor:
    """Free tensor product a * b."""
    _check_basis_compat(a.basis, b.basis)
    result = _zeros_like(a.data)
    _internals.dense_ft_fma(result, a.data, b.data, a.basis, rhs_depth=b.basis.depth)
    return DenseFreeTensor(result, a.basis)


def ft_inplace_mul(a: FreeTensor, b: FreeTensor, **kwargs):
    """a = a * b in place."""
    _check_basis_compat(a.basis, b.basis)
    _internals.dense_ft_inplace_mul(a.data, b.data, a.basis, b.basis.depth)


def antipode(a: FreeTensor, **kwargs) -> FreeTensor:
    """Antipode (signed word reversal) of a free tensor."""
    result = _zeros_like(a.data)
    _internals.dense_ft_antipode(result, a.data, a.basis)
    return FreeTensor(result, a.basis)


def ft_exp(x: FreeTensor, out_basis: TensorBasis | None = None) -> FreeTensor:
    """Tensor exponential (level 0 of x ignored)."""
    out_basis = out_basis or x.basis
    _check_basis_compat(out_basis, x.basis)
    _float_dtype(x.data)
    result = _zeros_like(x.data, out_basis.size())
    _internals.dense_ft_exp(result, x.data, out_basis)
    return FreeTensor(result, out_basis)


def ft_log(x: FreeTensor, out_basis: TensorBasis | None = None) -> FreeTensor:
    """Tensor logarithm (x assumed to have unit level 0); float64 series on the GPU."""
    out_basis = out_basis or x.basis
    _check_basis_compat(out_basis, x.basis)
    _float_dtype(x.data)
    result = _zeros_like(x.data, out_basis.size())
    _internals.dense_ft_log(result, x.data, out_basis)
    return FreeTensor(result, out_basis)


def ft_fmexp(multiplier: FreeTensor, exponent: FreeTensor,
             out_basis: TensorBasis | None = None) -> FreeTensor:
    """Fused multiply-exponential multiplier * exp(exponent)."""
    out_basis = out_basis or multiplier.basis
    _check_basis_compat(out_basis, multiplier.basis, exponent.basis)
    _float_dtype(multiplier.data)
    result = _zeros_like(multiplier.data, out_basis.size())
    _internals.dense_ft_fmexp(result, multiplier.data, exponent.data, out_basis)
    return FreeTensor(result, out_basis)


def ft_adjoint_left_mul(op: FreeTensor, arg: ShuffleTensor) -> ShuffleTensor:
    """Adjoint of left multiplication by op, applied to the shuffle tensor arg."""
    _check_basis_compat(op.basis, arg.basis)
    result = _zeros_like(arg.data)
    _internals.dense_ft_adjoint_left_mul(result, op.data, arg.data, op.basis, arg.basis.depth,
                                         op.basis.depth, arg.basis.depth)
    return ShuffleTensor(result, arg.basis)


def lie_to_tensor(arg: Lie, tensor_basis: TensorBasis | None = None,
                  scale_factor=None) -> FreeTensor:
    """Embed a Lie element (Hall basis coordinates) in the tensor algebra."""
    l2t = arg.basis.get_l2t_matrix(np.float64)
    tensor_basis = tensor_basis or TensorBasis(arg.basis.width, arg.basis.depth)
    result = _zeros_like(arg.data, tensor_basis.size())
    _internals.dense_lie_to_tensor(result, arg.data, l2t, arg.basis, tensor_basis,
                                   scale_factor=scale_factor)
    return FreeTensor(result, tensor_basis)


def tensor_to_lie(arg: FreeTensor, lie_basis: LieBasis | None = None,
                  scale_factor=None) -> Lie:
    """Project a free tensor onto the Lie algebra (Dynkin map in the Hall basis)."""
    lie_basis = lie_basis or LieBasis(arg.basis.width, arg.basis.depth)
    t2l = lie_basis.get_t2l_matrix(np.float64)
    result = _zeros_like(arg.data, lie_basis.size())
    _internals.dense_tensor_to_lie(result, arg.data, t2l, lie_basis, arg.basis,
                                   scale_factor=scale_factor)
    return Lie(result, lie_basis)
