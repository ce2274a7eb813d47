"""Host logic of the LieGroup layer (no kernel calls): constructors, shapes,
conversions between groups and broadcasting of operands."""

import pytest
import torch

from vipe_b200 import lietorch as LT


def test_identity_shapes_and_values():
    X = LT.SE3.Identity(2, 3, dtype=torch.float64)
    assert X.shape == (2, 3) and X.data.shape == (2, 3, 7)
    assert torch.equal(X.data[1, 2], LT.SE3.id_elem.double())
    assert LT.Sim3.Identity((4,)).data.shape == (4, 8)
    assert LT.SO3.IdentityLike(LT.SO3.Identity(5)).shape == (5,)


def test_group_conversions():
    R = LT.SO3(torch.tensor([[0.0, 0.0, 0.6, 0.8]]))
    T = LT.SE3(R)
    assert torch.equal(T.data, torch.tensor([[0.0, 0.0, 0.0, 0.0, 0.0, 0.6, 0.8]]))
    S = LT.Sim3(T)
    assert S.data.shape == (1, 8) and float(S.data[0, 7]) == 1.0
    assert LT.SO3(T).data.shape == (1, 4)
    assert LT.RxSO3(S).data.shape == (1, 5)
    with pytest.raises(ValueError):
        LT.SE3(torch.zeros(3, 8))


def test_broadcast_inputs():
    x = torch.randn(4, 1, 7)
    y = torch.randn(1, 5, 3)
    (x1, y1), shape = LT.broadcast_inputs(x, y)
    assert shape == (4, 5) and x1.shape == (20, 7) and y1.shape == (20, 3)
    assert torch.equal(x1.view(4, 5, 7)[:, 2], x[:, 0]) and torch.equal(y1.view(4, 5, 3)[3], y[0])
    (z,), s = LT.broadcast_inputs(torch.randn(2, 3, 6), None)
    assert s == (2, 3) and z.shape == (6, 6)


def test_indexing_view_and_cat():
    X = LT.SE3.Identity(6)
    assert X[2:4].shape == (2,)
    assert X.view((2, 3)).shape == (2, 3)
    assert LT.cat([X, X], 0).shape == (12,)
    Y = LT.SE3.Identity(6)
    Y[1] = LT.SE3(torch.tensor([1.0, 2, 3, 0, 0, 0, 1]))
    assert float(Y.data[1, 0]) == 1.0
