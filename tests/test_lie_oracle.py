"""CPU checks of the Lie-group oracle (oracle/lie.py) — axioms and finite differences.

The reference ships no lietorch test, so the oracle is pinned by properties:
exp/log round trips, X * X^-1 = I, Adj consistency (X Exp(a) X^-1 = Exp(Adj a)),
and the backward formulas against central finite differences where the
reference's formula is an exact derivative.
"""

import math

import numpy as np
import pytest

import oracle.lie as L

GROUPS = [1, 2, 3, 4]


def rand_tangent(gid, rng, scale=0.4):
    N, K = L.DIMS[gid]
    return rng.normal(0, scale, K)


@pytest.mark.parametrize("gid", GROUPS)
def test_exp_log_roundtrip(gid):
    rng = np.random.default_rng(gid)
    for _ in range(20):
        a = rand_tangent(gid, rng)
        np.testing.assert_allclose(L.exp(gid, a).log(), a, atol=1e-10)
    # tiny angles take the series branches
    a = rand_tangent(gid, rng, 1e-8)
    np.testing.assert_allclose(L.exp(gid, a).log(), a, atol=1e-14)


@pytest.mark.parametrize("gid", GROUPS)
def test_inverse_and_mul(gid):
    rng = np.random.default_rng(10 + gid)
    X = L.exp(gid, rand_tangent(gid, rng))
    Y = L.exp(gid, rand_tangent(gid, rng))
    I = X.mul(X.inv())
    np.testing.assert_allclose(I.log(), np.zeros(L.DIMS[gid][1]), atol=1e-12)
    p = rng.normal(size=3)
    np.testing.assert_allclose(X.mul(Y).act(p), X.act(Y.act(p)), atol=1e-12)


@pytest.mark.parametrize("gid", GROUPS)
def test_adjoint_identity(gid):
    rng = np.random.default_rng(20 + gid)
    X = L.exp(gid, rand_tangent(gid, rng))
    a = rand_tangent(gid, rng, 0.1)
    lhs = X.mul(L.exp(gid, a)).mul(X.inv())
    rhs = L.exp(gid, X.Adj() @ a)
    np.testing.assert_allclose(lhs.log(), rhs.log(), atol=1e-10)


@pytest.mark.parametrize("gid", [1, 2, 3])
def test_left_jacobian_is_exp_derivative(gid):
    # Exp(a + d) ~= Exp(J(a) d) Exp(a): J is the exact left Jacobian for SO3/RxSO3/SE3
    rng = np.random.default_rng(30 + gid)
    a = rand_tangent(gid, rng)
    K = L.DIMS[gid][1]
    J = L.left_jac(gid, a)
    h = 1e-6
    for k in range(K):
        d = np.zeros(K)
        d[k] = h
        num = (L.exp(gid, a + d).mul(L.exp(gid, a).inv()).log() - L.exp(gid, a - d).mul(L.exp(gid, a).inv()).log()) / (2 * h)
        np.testing.assert_allclose(num, J[:, k], atol=1e-6)
    np.testing.assert_allclose(L.left_jac_inv(gid, a) @ J, np.eye(K), atol=1e-10)


def test_sim3_left_jacobian_series_truncation():
    # the reference truncates the Sim3 series after ad^4/120 (sim3.h:160-170)
    a = np.array([0.1, -0.2, 0.05, 0.02, -0.03, 0.01, 0.04])
    X = L.ad(4, a)
    full = sum(np.linalg.matrix_power(X, k) / math.factorial(k + 1) for k in range(12))
    trunc = L.left_jac(4, a)
    assert np.abs(full - trunc).max() < 1e-6


@pytest.mark.parametrize("gid", GROUPS)
def test_act_backward_matches_fd(gid):
    rng = np.random.default_rng(40 + gid)
    N, K = L.DIMS[gid]
    X = L.exp(gid, rand_tangent(gid, rng)).data()[None]
    p = rng.normal(size=(1, 3))
    g = rng.normal(size=(1, 3))
    dX, dp = L.act_backward(gid, g, X, p)
    h = 1e-6
    for k in range(K):
        d = np.zeros(K)
        d[k] = h
        Xp = L.exp(gid, d).mul(L.Group(gid, X[0])).data()[None]
        Xm = L.exp(gid, -d).mul(L.Group(gid, X[0])).data()[None]
        num = (g * (L.act(gid, Xp, p) - L.act(gid, Xm, p))).sum() / (2 * h)
        assert abs(num - dX[0, k]) < 1e-6
    for k in range(3):
        d = np.zeros((1, 3))
        d[0, k] = h
        num = (g * (L.act(gid, X, p + d) - L.act(gid, X, p - d))).sum() / (2 * h)
        assert abs(num - dp[0, k]) < 1e-6
