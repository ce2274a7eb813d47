"""FP64 numpy restatement of the lietorch group ops — TEST INFRASTRUCTURE ONLY.

Follows the reference's group math (vipe csrc/lietorch_ext/so3.h:96-184,
rxso3.h:17-313 incl. calcW :184, se3.h:40-207 incl. calcQ, sim3.h:21-196 incl.
the truncated left-Jacobian series at :160-170) and the op conventions of
lietorch_gpu.cu:24-298 (gradient strides, output shapes).  Per-element Python
loops: meant for test-sized batches.

Parity is unpinned by reference tests (the reference ships no lietorch test);
the oracle is cross-checked by group axioms (exp/log round trips, inverse,
Adj consistency) and central finite differences in tests/test_lie_oracle.py.
"""

from __future__ import annotations

import numpy as np

EPS = 1e-6
DIMS = {1: (4, 3), 2: (5, 4), 3: (7, 6), 4: (8, 7)}


def hat(v):
    return np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])


def qnorm(q):
    return q / np.linalg.norm(q)


def qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + ax * bw + ay * bz - az * by, aw * by + ay * bw + az * bx - ax * bz,
                     aw * bz + az * bw + ax * by - ay * bx, aw * bw - ax * bx - ay * by - az * bz])


def qmat(q):
    x, y, z, w = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
    ])


def so3_exp(phi):
    t2 = phi @ phi
    t = np.sqrt(t2)
    if t < EPS:
        im = 0.5 - t2 / 48.0 + t2 * t2 / 3840.0
        re = 1.0 - t2 / 8.0 + t2 * t2 / 384.0
    else:
        im = np.sin(0.5 * t) / t
        re = np.cos(0.5 * t)
    return qnorm(np.array([im * phi[0], im * phi[1], im * phi[2], re]))


def so3_log(q):
    v, w = q[:3], q[3]
    n2 = v @ v
    if n2 < EPS * EPS:
        f = 2.0 / w - (2.0 / 3.0) * n2 / (w ** 3)
    else:
        n = np.sqrt(n2)
        if abs(w) < EPS:
            f = (np.pi if w > 0 else -np.pi) / n
        else:
            f = 2.0 * np.arctan(n / w) / n
    return f * v


def so3_J(phi):
    P = hat(phi)
    t2 = phi @ phi
    t = np.sqrt(t2)
    c1 = 0.5 - t2 / 24.0 if t < EPS else (1 - np.cos(t)) / t2
    c2 = 1.0 / 6.0 - t2 / 120.0 if t < EPS else (t - np.sin(t)) / (t2 * t)
    return np.eye(3) + c1 * P + c2 * P @ P


def so3_Jinv(phi):
    P = hat(phi)
    t = np.sqrt(phi @ phi)
    c2 = 1.0 / 12.0 if t < EPS else (1 - t * np.cos(0.5 * t) / (2 * np.sin(0.5 * t))) / (t * t)
    return np.eye(3) - 0.5 * P + c2 * P @ P


def quat_proj(q):
    J = np.zeros((4, 4))
    J[:3, :3] = 0.5 * (q[3] * np.eye(3) + hat(-q[:3]))
    J[3, :3] = 0.5 * (-q[:3])
    return J


def calcQ(a):
    T, P = hat(a[:3]), hat(a[3:6])
    th = np.linalg.norm(a[3:6])
    t2 = th * th
    t4 = t2 * t2
    c1 = 1 / 6 - t2 / 120 if th < EPS else (th - np.sin(th)) / (t2 * th)
    c2 = 1 / 24 - t2 / 720 if th < EPS else (t2 + 2 * np.cos(th) - 2) / (2 * t4)
    c3 = 1 / 120 - t2 / 2520 if th < EPS else (2 * th - 3 * np.sin(th) + th * np.cos(th)) / (2 * t4 * th)
    return (0.5 * T + c1 * (P @ T + T @ P + P @ T @ P) + c2 * (P @ P @ T + T @ P @ P - 3 * P @ T @ P)
            + c3 * (P @ T @ P @ P + P @ P @ T @ P))


def calcW(ps):
    phi, sig = ps[:3], ps[3]
    th = np.linalg.norm(phi)
    P = hat(phi)
    P2 = P @ P
    sc = np.exp(sig)
    if abs(sig) < EPS:
        C = 1.0
        if abs(th) < EPS:
            A, B = 0.5, 1.0 / 6.0
        else:
            A = (1 - np.cos(th)) / (th * th)
            B = (th - np.sin(th)) / (th ** 3)
    else:
        C = (sc - 1) / sig
        if abs(th) < EPS:
            s2 = sig * sig
            A = ((sig - 1) * sc + 1) / s2
            B = (sc * 0.5 * s2 + sc - 1 - sig * sc) / (s2 * sig)
        else:
            a = sc * np.sin(th)
            b = sc * np.cos(th)
            c = th * th + sig * sig
            A = (a * sig + (1 - b) * th) / (th * c)
            B = (C - ((b - 1) * sig + a * th) / c) / (th * th)
    return A * P + B * P2 + C * np.eye(3)


class Group:
    """Element of group `gid` with a normalised quaternion (as the reference loads it)."""

    def __init__(self, gid, data):
        self.gid = gid
        d = np.asarray(data, dtype=np.float64)
        if gid == 1:
            self.t, self.q, self.s = np.zeros(3), qnorm(d[:4]), 1.0
        elif gid == 2:
            self.t, self.q, self.s = np.zeros(3), qnorm(d[:4]), d[4]
        elif gid == 3:
            self.t, self.q, self.s = d[:3].copy(), qnorm(d[3:7]), 1.0
        else:
            self.t, self.q, self.s = d[:3].copy(), qnorm(d[3:7]), d[7]

    @classmethod
    def make(cls, gid, t, q, s):
        g = cls.__new__(cls)
        g.gid, g.t, g.q, g.s = gid, np.asarray(t, float), np.asarray(q, float), float(s)
        return g

    def data(self):
        if self.gid == 1:
            return self.q.copy()
        if self.gid == 2:
            return np.concatenate([self.q, [self.s]])
        if self.gid == 3:
            return np.concatenate([self.t, self.q])
        return np.concatenate([self.t, self.q, [self.s]])

    # --- core
    def R(self):
        return qmat(self.q)

    def sR(self):
        return self.s * qmat(self.q)

    def inv(self):
        qi = self.q * np.array([-1, -1, -1, 1.0])
        si = 1.0 / self.s
        ti = -(si * qmat(qi) @ self.t)
        return Group.make(self.gid, ti, qi, si)

    def mul(self, o):
        return Group.make(self.gid, self.t + self.sR() @ o.t, qnorm(qmul(self.q, o.q)), self.s * o.s)

    def act(self, p):
        return self.sR() @ p + self.t

    def act4(self, p):
        return np.concatenate([self.sR() @ p[:3] + self.t * p[3], [p[3]]])

    def mat4(self):
        T = np.eye(4)
        T[:3, :3] = self.sR()
        T[:3, 3] = self.t
        return T

    def Adj(self):
        g, R = self.gid, self.R()
        if g == 1:
            return R
        if g == 2:
            A = np.eye(4)
            A[:3, :3] = R
            return A
        if g == 3:
            A = np.zeros((6, 6))
            A[:3, :3] = R
            A[:3, 3:] = hat(self.t) @ R
            A[3:, 3:] = R
            return A
        A = np.eye(7)
        A[:3, :3] = self.sR()
        A[:3, 3:6] = hat(self.t) @ R
        A[:3, 6] = -self.t
        A[3:6, 3:6] = R
        return A

    def projector(self):
        g = self.gid
        if g == 1:
            return quat_proj(self.q)
        if g == 2:
            J = np.zeros((5, 5))
            J[:4, :4] = quat_proj(self.q)
            J[4, 3] = self.s
            return J
        if g == 3:
            J = np.zeros((7, 7))
            J[:3, :3] = np.eye(3)
            J[:3, 3:6] = hat(-self.t)
            J[3:7, 3:7] = quat_proj(self.q)
            return J
        J = np.zeros((8, 8))
        J[:3, :3] = np.eye(3)
        J[:3, 3:6] = hat(-self.t)
        J[:3, 6] = self.t
        J[3:7, 3:7] = quat_proj(self.q)
        J[7, 6] = self.s
        return J

    def log(self):
        g = self.gid
        phi = so3_log(self.q)
        if g == 1:
            return phi
        if g == 2:
            return np.concatenate([phi, [np.log(self.s)]])
        if g == 3:
            return np.concatenate([so3_Jinv(phi) @ self.t, phi])
        ps = np.concatenate([phi, [np.log(self.s)]])
        return np.concatenate([np.linalg.inv(calcW(ps)) @ self.t, ps])


def exp(gid, a):
    a = np.asarray(a, float)
    if gid == 1:
        return Group.make(1, np.zeros(3), so3_exp(a), 1.0)
    if gid == 2:
        return Group.make(2, np.zeros(3), so3_exp(a[:3]), np.exp(a[3]))
    if gid == 3:
        return Group.make(3, so3_J(a[3:6]) @ a[:3], so3_exp(a[3:6]), 1.0)
    return Group.make(4, calcW(a[3:7]) @ a[:3], so3_exp(a[3:6]), np.exp(a[6]))


def ad(gid, a):
    if gid == 1:
        return hat(a)
    if gid == 2:
        A = np.zeros((4, 4))
        A[:3, :3] = hat(a[:3])
        return A
    if gid == 3:
        A = np.zeros((6, 6))
        A[:3, :3] = hat(a[3:6])
        A[:3, 3:] = hat(a[:3])
        A[3:, 3:] = hat(a[3:6])
        return A
    A = np.zeros((7, 7))
    A[:3, :3] = hat(a[3:6]) + a[6] * np.eye(3)
    A[:3, 3:6] = hat(a[:3])
    A[:3, 6] = -a[:3]
    A[3:6, 3:6] = hat(a[3:6])
    return A


def left_jac(gid, a):
    if gid == 1:
        return so3_J(a)
    if gid == 2:
        J = np.eye(4)
        J[:3, :3] = so3_J(a[:3])
        return J
    if gid == 3:
        J = np.zeros((6, 6))
        J[:3, :3] = so3_J(a[3:6])
        J[:3, 3:] = calcQ(a)
        J[3:, 3:] = so3_J(a[3:6])
        return J
    X = ad(4, a)
    X2 = X @ X
    return np.eye(7) + X / 2 + X2 / 6 + X @ X2 / 24 + X2 @ X2 / 120


def left_jac_inv(gid, a):
    if gid == 1:
        return so3_Jinv(a)
    if gid == 2:
        J = np.eye(4)
        J[:3, :3] = so3_Jinv(a[:3])
        return J
    if gid == 3:
        Ji = so3_Jinv(a[3:6])
        J = np.zeros((6, 6))
        J[:3, :3] = Ji
        J[:3, 3:] = -Ji @ calcQ(a) @ Ji
        J[3:, 3:] = Ji
        return J
    X = ad(4, a)
    X2 = X @ X
    return np.eye(7) - X / 2 + X2 / 12 - X2 @ X2 / 720


def act_jac(gid, p):
    H = hat(-p)
    if gid == 1:
        return H
    if gid == 2:
        return np.concatenate([H, p[:, None]], 1)
    if gid == 3:
        return np.concatenate([np.eye(3), H], 1)
    return np.concatenate([np.eye(3), H, p[:, None]], 1)


def act4_jac(gid, p):
    N, K = DIMS[gid]
    J = np.zeros((4, K))
    H = hat(-p[:3])
    if gid == 1:
        J[:3, :3] = H
    elif gid == 2:
        J[:3, :3] = H
        J[:3, 3] = p[:3]
    elif gid == 3:
        J[:3, :3] = p[3] * np.eye(3)
        J[:3, 3:6] = H
    else:
        J[:3, :3] = p[3] * np.eye(3)
        J[:3, 3:6] = H
        J[:3, 6] = p[:3]
    return J


# ---------------------------------------------------------------- ops with the extension's shapes

def _rows(x):
    return np.asarray(x, dtype=np.float64)


def expm(gid, a):
    return np.stack([exp(gid, r).data() for r in _rows(a)])


def expm_backward(gid, grad, a):
    N, K = DIMS[gid]
    return np.stack([g[:K] @ left_jac(gid, r) for g, r in zip(_rows(grad), _rows(a))])


def logm(gid, X):
    return np.stack([Group(gid, x).log() for x in _rows(X)])


def logm_backward(gid, grad, X):
    N, K = DIMS[gid]
    out = np.zeros((len(X), N))
    for i, (g, x) in enumerate(zip(_rows(grad), _rows(X))):
        out[i, :K] = g @ left_jac_inv(gid, Group(gid, x).log())
    return out


def inv(gid, X):
    return np.stack([Group(gid, x).inv().data() for x in _rows(X)])


def inv_backward(gid, grad, X):
    N, K = DIMS[gid]
    out = np.zeros((len(X), N))
    for i, (g, x) in enumerate(zip(_rows(grad), _rows(X))):
        out[i, :K] = -(g[:K] @ Group(gid, x).inv().Adj())
    return out


def mul(gid, X, Y):
    return np.stack([Group(gid, x).mul(Group(gid, y)).data() for x, y in zip(_rows(X), _rows(Y))])


def mul_backward(gid, grad, X, Y):
    N, K = DIMS[gid]
    dX = np.zeros((len(X), N))
    dY = np.zeros((len(X), N))
    for i, (g, x) in enumerate(zip(_rows(grad), _rows(X))):
        dX[i, :K] = g[:K]
        dY[i, :K] = g[:K] @ Group(gid, x).Adj()
    return dX, dY


def adj(gid, X, a):
    return np.stack([Group(gid, x).Adj() @ v for x, v in zip(_rows(X), _rows(a))])


def adj_backward(gid, grad, X, a):
    N, K = DIMS[gid]
    dX = np.zeros((len(X), N))
    da = np.zeros((len(X), K))
    for i, (g, x, v) in enumerate(zip(_rows(grad), _rows(X), _rows(a))):
        A = Group(gid, x).Adj()
        da[i] = g @ A
        dX[i, :K] = -(g @ ad(gid, A @ v))
    return dX, da


def adjT(gid, X, a):
    return np.stack([Group(gid, x).Adj().T @ v for x, v in zip(_rows(X), _rows(a))])


def adjT_backward(gid, grad, X, a):
    N, K = DIMS[gid]
    dX = np.zeros((len(X), N))
    da = np.zeros((len(X), K))
    for i, (g, x, v) in enumerate(zip(_rows(grad), _rows(X), _rows(a))):
        A = Group(gid, x).Adj()
        da[i] = A @ g
        dX[i, :K] = -(v @ ad(gid, A @ g))
    return dX, da


def act(gid, X, p):
    return np.stack([Group(gid, x).act(v) for x, v in zip(_rows(X), _rows(p))])


def act_backward(gid, grad, X, p):
    N, K = DIMS[gid]
    dX = np.zeros((len(X), N))
    dp = np.zeros((len(X), 3))
    for i, (g, x, v) in enumerate(zip(_rows(grad), _rows(X), _rows(p))):
        G = Group(gid, x)
        dp[i] = g @ G.sR()
        dX[i, :K] = g @ act_jac(gid, G.act(v))
    return dX, dp


def act4(gid, X, p):
    return np.stack([Group(gid, x).act4(v) for x, v in zip(_rows(X), _rows(p))])


def act4_backward(gid, grad, X, p):
    N, K = DIMS[gid]
    dX = np.zeros((len(X), N))
    dp = np.zeros((len(X), 4))
    for i, (g, x, v) in enumerate(zip(_rows(grad), _rows(X), _rows(p))):
        G = Group(gid, x)
        dp[i] = g @ G.mat4()
        dX[i, :K] = g @ act4_jac(gid, G.act4(v))
    return dX, dp


def as_matrix(gid, X):
    return np.stack([Group(gid, x).mat4() for x in _rows(X)])


def projector(gid, X):
    return np.stack([Group(gid, x).projector() for x in _rows(X)])


def Jinv(gid, X, a):
    return np.stack([left_jac_inv(gid, Group(gid, x).log()) @ v for x, v in zip(_rows(X), _rows(a))])
