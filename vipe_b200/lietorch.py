"""Lie-group tensors on the vipe_b200 lietorch kernels.

Same API as the reference's ``vipe.ext.lietorch`` package (vipe/ext/lietorch/
groups.py:14-325, group_ops.py:10-125, broadcasting.py:6-33) so that callers
(``SE3(poses).inv() * SE3(poses)``, ``.act``, ``.retr``, ``.log``, ``Sim3``, ...)
switch by import:

    from vipe_b200.lietorch import SE3, Sim3, SO3, RxSO3, LieGroupParameter, cat

A group object wraps a data tensor ``(..., embedded_dim)``; every operation
broadcasts the leading dimensions of its operands, flattens them into one batch
and calls the corresponding ``lietorch_ext`` kernel (group ids 1 SO3, 2 RxSO3,
3 SE3, 4 Sim3).  Each op is a ``torch.autograd.Function`` whose backward is the
kernel's hand-written backward; as in lietorch, the gradient with respect to a
group element is expressed in its tangent space (stored in the first
``manifold_dim`` entries of the data gradient).  ``InitFromVec`` / ``vec``
convert between that convention and Euclidean embedding gradients through the
projector kernel.
"""

from __future__ import annotations

import math

import torch

from .ext import lietorch_ext as _ext


# ---------------------------------------------------------------- autograd ops

def _make_op(name: str, fwd, bwd):
    """autograd.Function for one kernel: forward(group_id, *inputs) -> out."""

    def forward(ctx, group_id, *inputs):
        ctx.group_id = group_id
        ctx.save_for_backward(*inputs)
        return fwd(group_id, *inputs)

    def backward(ctx, grad):
        if bwd is None:
            raise RuntimeError(f"{name} has no backward in lietorch")
        grads = bwd(ctx.group_id, grad.contiguous(), *ctx.saved_tensors)
        return (None, *grads)

    return type(name, (torch.autograd.Function,), {"forward": staticmethod(forward),
                                                      "backward": staticmethod(backward)})


Exp = _make_op("Exp", _ext.expm, _ext.expm_backward)
Log = _make_op("Log", _ext.logm, _ext.logm_backward)
Inv = _make_op("Inv", _ext.inv, _ext.inv_backward)
Mul = _make_op("Mul", _ext.mul, _ext.mul_backward)
Adj = _make_op("Adj", _ext.adj, _ext.adj_backward)
AdjT = _make_op("AdjT", _ext.adjT, _ext.adjT_backward)
Act3 = _make_op("Act3", _ext.act, _ext.act_backward)
Act4 = _make_op("Act4", _ext.act4, _ext.act4_backward)
Jinv = _make_op("Jinv", _ext.Jinv, None)
ToMatrix = _make_op("ToMatrix", _ext.as_matrix, None)


class FromVec(torch.autograd.Function):
    """Embedding vector -> group data; backward maps an embedding gradient to the tangent one."""

    @staticmethod
    def forward(ctx, group_id, x):
        ctx.group_id = group_id
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, grad):
        (x,) = ctx.saved_tensors
        P = _ext.projector(ctx.group_id, x)  # (B, N, K)
        return None, (grad.unsqueeze(-2) @ torch.linalg.pinv(P)).squeeze(-2)


class ToVec(torch.autograd.Function):
    """Group data -> embedding vector; backward maps a tangent gradient to the embedding one."""

    @staticmethod
    def forward(ctx, group_id, x):
        ctx.group_id = group_id
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, grad):
        (x,) = ctx.saved_tensors
        P = _ext.projector(ctx.group_id, x)
        return None, (grad.unsqueeze(-2) @ P).squeeze(-2)


def broadcast_inputs(x, y):
    """Flattens x (and y, broadcasting their leading dims) into (B, d) rows; returns (rows, out_shape)."""
    if y is None:
        return (x.reshape(-1, x.shape[-1]).contiguous(),), tuple(x.shape[:-1])
    if x.dim() != y.dim():
        raise ValueError("lietorch broadcasting needs operands of equal rank")
    lead = torch.broadcast_shapes(x.shape[:-1], y.shape[:-1])
    x1 = x.expand(*lead, x.shape[-1]).reshape(-1, x.shape[-1]).contiguous()
    y1 = y.expand(*lead, y.shape[-1]).reshape(-1, y.shape[-1]).contiguous()
    return (x1, y1), tuple(lead)


# ---------------------------------------------------------------- groups

class LieGroup:
    """A batch of group elements stored as ``data`` (..., embedded_dim)."""

    group_name = ""
    group_id = 0
    manifold_dim = 0
    embedded_dim = 0
    id_elem = None

    def __init__(self, data: torch.Tensor):
        if data.shape[-1] != self.embedded_dim:
            raise ValueError(f"{self.group_name} data needs last dimension {self.embedded_dim}, got {data.shape[-1]}")
        self.data = data

    def __repr__(self):
        return f"{self.group_name} Group Object: {tuple(self.data.shape)}"

    # -- metadata
    @property
    def shape(self):
        return self.data.shape[:-1]

    @property
    def device(self):
        return self.data.device

    @property
    def dtype(self):
        return self.data.dtype

    def vec(self):
        return self.apply_op(ToVec, self.data)

    @property
    def tangent_shape(self):
        return self.data.shape[:-1] + (self.manifold_dim,)

    # -- constructors
    @staticmethod
    def _shape_arg(batch_shape):
        if len(batch_shape) == 1 and isinstance(batch_shape[0], (tuple, list, torch.Size)):
            return tuple(batch_shape[0])
        return tuple(batch_shape)

    @classmethod
    def Identity(cls, *batch_shape, **kwargs):
        shape = cls._shape_arg(batch_shape)
        data = cls.id_elem.to(device=kwargs.get("device"), dtype=kwargs.get("dtype", cls.id_elem.dtype))
        n = math.prod(shape) if shape else 1
        return cls(data.reshape(1, -1).repeat(n, 1)).view(shape)

    @classmethod
    def IdentityLike(cls, G):
        return cls.Identity(G.shape, device=G.data.device, dtype=G.data.dtype)

    @classmethod
    def InitFromVec(cls, data):
        return cls(cls.apply_op(FromVec, data))

    @classmethod
    def Random(cls, *batch_shape, sigma=1.0, **kwargs):
        shape = cls._shape_arg(batch_shape)
        xi = torch.randn(shape + (cls.manifold_dim,), **kwargs)
        return cls.exp(sigma * xi)

    @classmethod
    def apply_op(cls, op, x, y=None):
        inputs, out_shape = broadcast_inputs(x, y)
        out = op.apply(cls.group_id, *inputs)
        return out.view(out_shape + (-1,))

    # -- maps and products
    @classmethod
    def exp(cls, x):
        return cls(cls.apply_op(Exp, x))

    def quaternion(self):
        return self.data[..., :4] if self.group_id in (1, 2) else self.data[..., 3:7]

    def log(self):
        return self.apply_op(Log, self.data)

    def inv(self):
        return self.__class__(self.apply_op(Inv, self.data))

    def mul(self, other):
        return self.__class__(self.apply_op(Mul, self.data, other.data))

    def retr(self, a):
        """Exp(a) * X"""
        return self.__class__(self.apply_op(Mul, self.__class__.apply_op(Exp, a), self.data))

    def adj(self, a):
        return self.apply_op(Adj, self.data, a)

    def adjT(self, a):
        return self.apply_op(AdjT, self.data, a)

    def Jinv(self, a):
        return self.apply_op(Jinv, self.data, a)

    def act(self, p):
        if p.shape[-1] == 3:
            return self.apply_op(Act3, self.data, p)
        if p.shape[-1] == 4:
            return self.apply_op(Act4, self.data, p)
        raise ValueError("act needs points (..., 3) or homogeneous points (..., 4)")

    def matrix(self):
        """4x4 matrices, built by acting on the homogeneous basis."""
        eye = torch.eye(4, dtype=self.dtype, device=self.device)
        eye = eye.view([1] * (self.data.dim() - 1) + [4, 4])
        return self.__class__(self.data[..., None, :]).act(eye).transpose(-1, -2)

    def translation(self):
        p = torch.tensor([0.0, 0.0, 0.0, 1.0], dtype=self.dtype, device=self.device)
        return self.apply_op(Act4, self.data, p.view([1] * (self.data.dim() - 1) + [4]))

    # -- tensor-like plumbing
    def detach(self):
        return self.__class__(self.data.detach())

    def view(self, dims):
        return self.__class__(self.data.view(tuple(dims) + (self.embedded_dim,)))

    def __mul__(self, other):
        if isinstance(other, LieGroup):
            return self.mul(other)
        if isinstance(other, torch.Tensor):
            return self.act(other)
        return NotImplemented

    def __getitem__(self, index):
        return self.__class__(self.data[index])

    def __setitem__(self, index, item):
        self.data[index] = item.data

    def to(self, *args, **kwargs):
        return self.__class__(self.data.to(*args, **kwargs))

    def cpu(self):
        return self.__class__(self.data.cpu())

    def cuda(self):
        return self.__class__(self.data.cuda())

    def float(self, device=None):
        return self.__class__(self.data.float())

    def double(self, device=None):
        return self.__class__(self.data.double())

    def unbind(self, dim=0):
        return [self.__class__(x) for x in self.data.unbind(dim=dim)]


class SO3(LieGroup):
    group_name, group_id, manifold_dim, embedded_dim = "SO3", 1, 3, 4
    id_elem = torch.tensor([0.0, 0.0, 0.0, 1.0])

    def __init__(self, data):
        if isinstance(data, SE3):
            data = data.data[..., 3:7]
        super().__init__(data)


class RxSO3(LieGroup):
    group_name, group_id, manifold_dim, embedded_dim = "RxSO3", 2, 4, 5
    id_elem = torch.tensor([0.0, 0.0, 0.0, 1.0, 1.0])

    def __init__(self, data):
        if isinstance(data, Sim3):
            data = data.data[..., 3:8]
        super().__init__(data)


class SE3(LieGroup):
    group_name, group_id, manifold_dim, embedded_dim = "SE3", 3, 6, 7
    id_elem = torch.tensor([0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0])

    def __init__(self, data):
        if isinstance(data, SO3):
            t = torch.zeros_like(data.data[..., :3])
            data = torch.cat([t, data.data], -1)
        super().__init__(data)

    def scale(self, s):
        t, q = self.data.split([3, 4], -1)
        return SE3(torch.cat([t * s.unsqueeze(-1), q], -1))


class Sim3(LieGroup):
    group_name, group_id, manifold_dim, embedded_dim = "Sim3", 4, 7, 8
    id_elem = torch.tensor([0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0])

    def __init__(self, data):
        if isinstance(data, SO3):
            data = torch.cat([torch.zeros_like(data.data[..., :3]), data.data, torch.ones_like(data.data[..., :1])], -1)
        elif isinstance(data, SE3):
            data = torch.cat([data.data, torch.ones_like(data.data[..., :1])], -1)
        elif isinstance(data, RxSO3):
            data = torch.cat([torch.zeros_like(data.data[..., :3]), data.data], -1)
        super().__init__(data)


class LieGroupParameter(torch.Tensor):
    """Optimisable group element: a tensor of the group's data whose gradient is a
    tangent gradient; ``add_(update, alpha)`` retracts instead of adding."""

    from torch._C import _disabled_torch_function_impl

    __torch_function__ = _disabled_torch_function_impl

    def __new__(cls, group, requires_grad=True):
        data = torch.zeros(group.tangent_shape, device=group.data.device, dtype=group.data.dtype)
        return torch.Tensor._make_subclass(cls, data, requires_grad)

    def __init__(self, group):
        self.group = group

    def retr(self):
        return self.group.retr(self)

    def log(self):
        return self.retr().log()

    def inv(self):
        return self.retr().inv()

    def adj(self, a):
        return self.retr().adj(a)

    def __mul__(self, other):
        if isinstance(other, LieGroupParameter):
            return self.retr() * other.retr()
        return self.retr() * other

    def add_(self, update, alpha):
        self.group = self.group.exp(alpha * update) * self.group

    def __getitem__(self, index):
        return self.retr().__getitem__(index)


def cat(group_list, dim):
    """Concatenates group objects of one type along a batch dimension."""
    return group_list[0].__class__(torch.cat([X.data for X in group_list], dim=dim))
