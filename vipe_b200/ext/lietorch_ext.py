"""lietorch_ext — drop-in for the reference's ``vipe.ext.lietorch_ext`` pybind module.

Reference bindings: vipe csrc/lietorch_ext/lietorch.cpp:306-336 (19 functions),
host allocation in lietorch_gpu.cu:303-562.  Group ids: 1 SO3, 2 RxSO3, 3 SE3,
4 Sim3.  Inputs are (B, N) group elements / (B, K) tangents / (B, 3|4) points in
float32 or float64; outputs have the reference's shapes.  Gradients with
respect to group elements are (B, N) tensors whose first K columns hold the
tangent-space gradient (reference convention).

Only CUDA tensors are supported (the reference also has a CPU path; callers on
this hot path keep their tensors on the GPU).
"""

from __future__ import annotations

import torch

from .. import _lib

# (N embedding, K tangent) per group id
DIMS = {1: (4, 3), 2: (5, 4), 3: (7, 6), 4: (8, 7)}


def _prep(group_index, *tensors):
    if group_index not in DIMS:
        raise RuntimeError(f"unsupported group index {group_index}")
    dt = None
    for i, t in enumerate(tensors):
        _lib.require_cuda(f"input {i}", t)
        _lib.require_contiguous(f"input {i}", t)
        if dt is None:
            dt = t.dtype
    if dt not in (torch.float32, torch.float64):
        raise RuntimeError(f"lietorch_ext supports float32 and float64, got {dt}")
    for t in tensors:
        if t.dtype != dt:
            raise RuntimeError("all inputs must share one dtype")
    return DIMS[group_index], _lib.DTYPE_CODE[dt]


def _call(fn, group_index, dtype_code, batch, ins, outs, stream_t):
    rc = getattr(_lib.load(), fn)(group_index, dtype_code, batch, *[t.data_ptr() for t in ins],
                                  *[t.data_ptr() for t in outs], _lib.stream_of(stream_t))
    _lib.check(rc, f"lietorch_ext.{fn[9:]}")


def expm(group_index, a):
    (N, K), dc = _prep(group_index, a)
    X = torch.zeros(a.shape[0], N, dtype=a.dtype, device=a.device)
    _call("vipe_lie_expm", group_index, dc, a.shape[0], [a], [X], a)
    return X


def expm_backward(group_index, grad, a):
    (N, K), dc = _prep(group_index, grad, a)
    da = torch.zeros(a.shape, dtype=grad.dtype, device=a.device)
    _call("vipe_lie_expm_backward", group_index, dc, a.shape[0], [grad, a], [da], a)
    return [da]


def logm(group_index, X):
    (N, K), dc = _prep(group_index, X)
    a = torch.zeros(X.shape[0], K, dtype=X.dtype, device=X.device)
    _call("vipe_lie_logm", group_index, dc, X.shape[0], [X], [a], X)
    return a


def logm_backward(group_index, grad, X):
    (N, K), dc = _prep(group_index, grad, X)
    dX = torch.zeros(X.shape, dtype=grad.dtype, device=X.device)
    _call("vipe_lie_logm_backward", group_index, dc, X.shape[0], [grad, X], [dX], X)
    return [dX]


def inv(group_index, X):
    (N, K), dc = _prep(group_index, X)
    Y = torch.zeros_like(X)
    _call("vipe_lie_inv", group_index, dc, X.shape[0], [X], [Y], X)
    return Y


def inv_backward(group_index, grad, X):
    (N, K), dc = _prep(group_index, grad, X)
    dX = torch.zeros(X.shape, dtype=grad.dtype, device=X.device)
    _call("vipe_lie_inv_backward", group_index, dc, X.shape[0], [grad, X], [dX], X)
    return [dX]


def mul(group_index, X, Y):
    (N, K), dc = _prep(group_index, X, Y)
    Z = torch.zeros_like(X)
    _call("vipe_lie_mul", group_index, dc, X.shape[0], [X, Y], [Z], X)
    return Z


def mul_backward(group_index, grad, X, Y):
    (N, K), dc = _prep(group_index, grad, X, Y)
    dX = torch.zeros(X.shape, dtype=grad.dtype, device=X.device)
    dY = torch.zeros(Y.shape, dtype=grad.dtype, device=X.device)
    _call("vipe_lie_mul_backward", group_index, dc, X.shape[0], [grad, X, Y], [dX, dY], X)
    return [dX, dY]


def adj(group_index, X, a):
    (N, K), dc = _prep(group_index, X, a)
    b = torch.zeros(a.shape, dtype=a.dtype, device=a.device)
    _call("vipe_lie_adj", group_index, dc, X.shape[0], [X, a], [b], X)
    return b


def adj_backward(group_index, grad, X, a):
    (N, K), dc = _prep(group_index, grad, X, a)
    dX = torch.zeros(X.shape, dtype=grad.dtype, device=X.device)
    da = torch.zeros(a.shape, dtype=grad.dtype, device=X.device)
    _call("vipe_lie_adj_backward", group_index, dc, X.shape[0], [grad, X, a], [dX, da], X)
    return [dX, da]


def adjT(group_index, X, a):
    (N, K), dc = _prep(group_index, X, a)
    b = torch.zeros(a.shape, dtype=a.dtype, device=a.device)
    _call("vipe_lie_adjT", group_index, dc, X.shape[0], [X, a], [b], X)
    return b


def adjT_backward(group_index, grad, X, a):
    (N, K), dc = _prep(group_index, grad, X, a)
    dX = torch.zeros(X.shape, dtype=grad.dtype, device=X.device)
    da = torch.zeros(a.shape, dtype=grad.dtype, device=X.device)
    _call("vipe_lie_adjT_backward", group_index, dc, X.shape[0], [grad, X, a], [dX, da], X)
    return [dX, da]


def act(group_index, X, p):
    (N, K), dc = _prep(group_index, X, p)
    q = torch.zeros(p.shape, dtype=p.dtype, device=p.device)
    _call("vipe_lie_act", group_index, dc, X.shape[0], [X, p], [q], X)
    return q


def act_backward(group_index, grad, X, p):
    (N, K), dc = _prep(group_index, grad, X, p)
    dX = torch.zeros(X.shape, dtype=grad.dtype, device=X.device)
    dp = torch.zeros(p.shape, dtype=grad.dtype, device=X.device)
    _call("vipe_lie_act_backward", group_index, dc, X.shape[0], [grad, X, p], [dX, dp], X)
    return [dX, dp]


def act4(group_index, X, p):
    (N, K), dc = _prep(group_index, X, p)
    q = torch.zeros(p.shape, dtype=p.dtype, device=p.device)
    _call("vipe_lie_act4", group_index, dc, X.shape[0], [X, p], [q], X)
    return q


def act4_backward(group_index, grad, X, p):
    (N, K), dc = _prep(group_index, grad, X, p)
    dX = torch.zeros(X.shape, dtype=grad.dtype, device=X.device)
    dp = torch.zeros(p.shape, dtype=grad.dtype, device=X.device)
    _call("vipe_lie_act4_backward", group_index, dc, X.shape[0], [grad, X, p], [dX, dp], X)
    return [dX, dp]


def as_matrix(group_index, X):
    (N, K), dc = _prep(group_index, X)
    T = torch.zeros(X.shape[0], 4, 4, dtype=X.dtype, device=X.device)
    _call("vipe_lie_as_matrix", group_index, dc, X.shape[0], [X], [T], X)
    return T


def projector(group_index, X):
    (N, K), dc = _prep(group_index, X)
    P = torch.zeros(X.shape[0], N, N, dtype=X.dtype, device=X.device)
    _call("vipe_lie_projector", group_index, dc, X.shape[0], [X], [P], X)
    return P


def Jinv(group_index, X, a):
    (N, K), dc = _prep(group_index, X, a)
    b = torch.zeros(a.shape, dtype=a.dtype, device=a.device)
    _call("vipe_lie_Jinv", group_index, dc, X.shape[0], [X, a], [b], X)
    return b
