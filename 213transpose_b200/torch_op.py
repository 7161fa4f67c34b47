"""PyTorch binding: ``torch.ops.t213.transpose_`` (registered on import).

``permute_(x, dims)`` is ``x.permute(dims).contiguous()`` done in place:
torch's dims (slowest first) are turned into the reference's rank-N
convention (fastest first) and handed to t213_permute, at most ndim - 1
in-place 213 transposes; x then has the permuted shape, contiguous.

``transpose_(x, dim0=-2, dim1=-1)`` swaps the two fastest dimensions of a
contiguous CUDA tensor in place: x of shape (..., d2, d1) is transposed slice
by slice through the C ABI (t213_transpose with d1 = x.size(-1),
d2 = x.size(-2), d3 = the product of the leading dimensions, on the tensor's
current stream) and its metadata becomes (..., d1, d2), contiguous.  The
reference's axes (d1, d2, d3) are torch's dims (-1, -2, leading), so its 213
permutation swaps torch dims -2 and -1; no other pair is accepted.  The
storage is not reallocated: views taken before the call see the transposed
bytes under their old shape.
"""
from __future__ import annotations

import math

import torch

from .api import permute as _permute
from .api import transpose as _transpose

_LIB = torch.library.Library("t213", "DEF")
_LIB.define("transpose_(Tensor(a!) self, int dim0=-2, int dim1=-1) -> Tensor(a!)")
_LIB.define("permute_(Tensor(a!) self, int[] dims) -> Tensor(a!)")


def _check_dims(x: torch.Tensor, dim0: int, dim1: int) -> None:
    if x.dim() < 2:
        raise ValueError("t213.transpose_ needs a tensor of at least 2 dimensions")
    d = sorted((dim0 % x.dim(), dim1 % x.dim()))
    if d != [x.dim() - 2, x.dim() - 1]:
        raise ValueError("t213.transpose_ swaps the last two dimensions (the reference's axes d1 and d2)")
    if not x.is_contiguous():
        raise ValueError("t213.transpose_ needs a contiguous tensor")


def _impl(x: torch.Tensor, dim0: int = -2, dim1: int = -1) -> torch.Tensor:
    _check_dims(x, dim0, dim1)
    d1, d2 = x.size(-1), x.size(-2)
    d3 = math.prod(x.shape[:-2])
    if x.numel():
        _transpose(x, d1, d2, d3)
    shape = tuple(x.shape[:-2]) + (d1, d2)
    return x.as_strided_(shape, torch.empty(shape, device="meta").stride())


torch.library.impl(_LIB, "transpose_", "CUDA")(_impl)


@torch.library.impl(_LIB, "transpose_", "CPU")
def _cpu(x: torch.Tensor, dim0: int = -2, dim1: int = -1) -> torch.Tensor:
    raise RuntimeError("t213.transpose_ runs on CUDA tensors only (no CPU path)")


@torch.library.register_fake("t213::transpose_")
def _fake(x: torch.Tensor, dim0: int = -2, dim1: int = -1) -> torch.Tensor:
    _check_dims(x, dim0, dim1)
    shape = tuple(x.shape[:-2]) + (x.size(-1), x.size(-2))
    return x.as_strided_(shape, torch.empty(shape, device="meta").stride())


def transpose_(x: torch.Tensor, dim0: int = -2, dim1: int = -1) -> torch.Tensor:
    """Same as torch.ops.t213.transpose_."""
    return torch.ops.t213.transpose_(x, dim0, dim1)


def _perm_args(x: torch.Tensor, dims):
    n = x.dim()
    p = [int(d) % n if n else 0 for d in dims]
    if sorted(p) != list(range(n)):
        raise ValueError("t213.permute_ needs a permutation of the tensor's dimensions")
    if not x.is_contiguous():
        raise ValueError("t213.permute_ needs a contiguous tensor")
    shape = tuple(x.shape[d] for d in p)
    return p, shape


@torch.library.impl(_LIB, "permute_", "CUDA")
def _permute_impl(x: torch.Tensor, dims) -> torch.Tensor:
    p, shape = _perm_args(x, dims)
    n = x.dim()
    if x.numel() and n > 1:
        # torch dim i (slowest first) is the reference's axis n-1-i (fastest
        # first); output axis j of the reference is input axis n-1-p[n-1-j]
        ref_dims = [x.size(n - 1 - a) for a in range(n)]
        ref_perm = [n - 1 - p[n - 1 - j] for j in range(n)]
        _permute(x, ref_dims, ref_perm)
    return x.as_strided_(shape, torch.empty(shape, device="meta").stride())


@torch.library.impl(_LIB, "permute_", "CPU")
def _permute_cpu(x: torch.Tensor, dims) -> torch.Tensor:
    raise RuntimeError("t213.permute_ runs on CUDA tensors only (no CPU path)")


@torch.library.register_fake("t213::permute_")
def _permute_fake(x: torch.Tensor, dims) -> torch.Tensor:
    _, shape = _perm_args(x, dims)
    return x.as_strided_(shape, torch.empty(shape, device="meta").stride())


def permute_(x: torch.Tensor, dims) -> torch.Tensor:
    """Same as torch.ops.t213.permute_."""
    return torch.ops.t213.permute_(x, list(dims))
