"""The LieGroup layer (vipe_b200.lietorch) on the GPU.

Values against the FP64 oracle (oracle/lie.py) for SO3, RxSO3, SE3 and Sim3
(atol 1e-9 in float64): exp, log, inv, mul, act on points and homogeneous points, retr, adj,
matrix, translation, with broadcasting of leading dimensions.  Gradients: torch's
gradcheck (float64, central differences) through compositions that start from
tangent vectors, so every op's backward is exercised in the tangent convention
the layer uses (exp, mul, inv, act, adj, log, retr, as in the reference's
lietorch group tests).
"""

import numpy as np
import pytest
import torch

import oracle.lie as L
from vipe_b200 import lietorch as LT

pytestmark = pytest.mark.gpu

GROUPS = [(LT.SE3, 3), (LT.Sim3, 4), (LT.SO3, 1), (LT.RxSO3, 2)]


def _rand_tangent(K, *shape, scale=0.5, seed=0):
    g = torch.Generator().manual_seed(seed)
    return (scale * torch.randn(*shape, K, generator=g, dtype=torch.float64)).cuda()


@pytest.mark.parametrize("cls, gid", GROUPS)
def test_values_against_oracle(cls, gid):
    K = cls.manifold_dim
    a = _rand_tangent(K, 6, seed=1)
    b = _rand_tangent(K, 6, seed=2)
    X, Y = cls.exp(a), cls.exp(b)
    ox = [L.exp(gid, r) for r in a.cpu().numpy()]
    oy = [L.exp(gid, r) for r in b.cpu().numpy()]
    np.testing.assert_allclose(X.data.cpu().numpy(), np.stack([g.data() for g in ox]), atol=1e-9)
    np.testing.assert_allclose(X.log().cpu().numpy(), a.cpu().numpy(), atol=1e-9)
    np.testing.assert_allclose(X.inv().data.cpu().numpy(), np.stack([g.inv().data() for g in ox]), atol=1e-9)
    np.testing.assert_allclose((X * Y).data.cpu().numpy(),
                               np.stack([L.mul(gid, x.data()[None], y.data()[None])[0] for x, y in zip(ox, oy)]),
                               atol=1e-9)
    p = torch.randn(6, 3, dtype=torch.float64).cuda()
    np.testing.assert_allclose((X * p).cpu().numpy(),
                               np.stack([L.act(gid, x.data()[None], q[None])[0] for x, q in zip(ox, p.cpu().numpy())]),
                               atol=1e-9)
    p4 = torch.cat([p, torch.rand(6, 1, dtype=torch.float64).cuda()], -1)
    np.testing.assert_allclose(X.act(p4).cpu().numpy(),
                               np.stack([L.act4(gid, x.data()[None], q[None])[0] for x, q in zip(ox, p4.cpu().numpy())]),
                               atol=1e-9)
    np.testing.assert_allclose(X.retr(b).data.cpu().numpy(), (cls.exp(b) * X).data.cpu().numpy(), atol=1e-12)
    np.testing.assert_allclose(X.adj(b).cpu().numpy(),
                               np.stack([L.adj(gid, x.data()[None], v[None])[0] for x, v in zip(ox, b.cpu().numpy())]),
                               atol=1e-9)
    M = X.matrix()
    assert M.shape == (6, 4, 4)
    hp = torch.cat([p, torch.ones(6, 1, dtype=torch.float64, device="cuda")], -1)
    np.testing.assert_allclose((M @ hp[..., None])[..., 0].cpu().numpy(), X.act(hp).cpu().numpy(), atol=1e-9)
    if gid in (3, 4):
        np.testing.assert_allclose(X.translation()[..., :3].cpu().numpy(), X.data[..., :3].cpu().numpy(), atol=1e-12)


def test_broadcasting_of_leading_dims():
    X = LT.SE3.exp(_rand_tangent(6, 4, 1, seed=3))
    Y = LT.SE3.exp(_rand_tangent(6, 1, 5, seed=4))
    Z = X * Y
    assert Z.shape == (4, 5)
    for i in range(4):
        for j in range(5):
            torch.testing.assert_close(Z.data[i, j], (X[i, 0] * Y[0, j]).data, rtol=0, atol=1e-12)
    pts = torch.randn(4, 5, 3, dtype=torch.float64, device="cuda")
    assert (X * pts).shape == (4, 5, 3)


# Sim3's exp backward reproduces the reference's truncated left-Jacobian series
# (csrc/lietorch_ext/sim3.h:168), exact only to O(|a|^5): small tangents there.
@pytest.mark.parametrize("cls, scale", [(LT.SE3, 0.5), (LT.Sim3, 0.05), (LT.SO3, 0.5), (LT.RxSO3, 0.5)])
def test_gradients_through_every_op(cls, scale):
    K = cls.manifold_dim
    a = _rand_tangent(K, 3, scale=scale, seed=5).requires_grad_(True)
    b = _rand_tangent(K, 3, scale=scale, seed=6).requires_grad_(True)
    p = torch.randn(3, 3, dtype=torch.float64, device="cuda", requires_grad=True)
    v = _rand_tangent(K, 3, seed=7).requires_grad_(True)

    def f(a, b, p, v):
        X, Y = cls.exp(a), cls.exp(b)
        Z = (X * Y.inv()).retr(0.1 * v)
        return torch.cat([Z.log(), Z.act(p), X.adj(v), Y.adjT(v)], -1)

    assert torch.autograd.gradcheck(f, (a, b, p, v), eps=1e-6, atol=1e-6, rtol=1e-5)


def test_parameter_and_cat():
    X = LT.SE3.exp(_rand_tangent(6, 2, seed=8))
    P = LT.LieGroupParameter(X)
    assert P.shape == (2, 6)
    torch.testing.assert_close(P.retr().data, X.data)
    P.add_(_rand_tangent(6, 2, seed=9), alpha=0.5)
    assert not torch.equal(P.group.data, X.data)
    C = LT.cat([X, X.inv()], 0)
    assert C.shape == (4,)
