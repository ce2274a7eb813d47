"""Dense, differentiable FP64 restatement of the fused BA in torch — TEST INFRASTRUCTURE ONLY.

Follows the same reference semantics as oracle/ba_oracle.cpp (vipe
csrc/slam_ext/geom_kernels.cu:178-524 per-edge math, :1626-1847 LM loop): 0.001
weight scale, MIN_DEPTH 0.25 validity mask, stereo edges (ii == jj) with the
fixed relative pose (-0.1, 0, 0) and no pose terms, C = 1 / w = 0 on inactive
depth frames, damping diag += ep + lm * diag of the reduced system, and the
back-substitution that leaves pose t0's rows out (geom_kernels.cu:1186).  The
reduced system is solved densely (torch.linalg.solve) instead of by Cholesky.

Written with torch ops only, so torch.autograd differentiates the whole solve,
including the second derivatives of the reprojection that the Jacobian formulas
carry.  ``detach_damping`` treats the LM damping ep + lm*diag(S) as a constant;
with it False (as the CUDA adjoint does) the damping's dependence on diag(S) is
differentiated as well.

Poses use lietorch's SE3 layout [tx ty tz qx qy qz qw] (world-to-camera), and
tangent vectors [tau, phi]; Sim3 poses (N, 8) [t q s] with tangents [tau, phi,
sigma] select the Sim3 form (no counterpart in the reference, whose fused BA is
SE3-only: the same residuals, weights and solver with 7x7 pose blocks); gradients with respect to poses are taken as left
tangent perturbations T -> Exp(eps) T (see ``perturb``).
"""

from __future__ import annotations

import torch

MIN_DEPTH = 0.25


def _cross(a, b):
    return torch.cross(a, b, dim=-1)


def quat_rot(q, x):
    v, w = q[..., :3], q[..., 3:4]
    uv = 2.0 * _cross(v, x)
    return x + w * uv + _cross(v, uv)


def quat_mul(a, b):
    ax, ay, az, aw = a.unbind(-1)
    bx, by, bz, bw = b.unbind(-1)
    return torch.stack([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                        aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz], -1)


def se3_exp(xi):
    """(..., 6) [tau, phi] -> (..., 7), as the reference's expSE3 (geom_kernels.cu:116-136):
    the translation series is applied only for theta > 1e-4."""
    tau, phi = xi[..., :3], xi[..., 3:]
    th2 = (phi * phi).sum(-1, keepdim=True)
    small = th2 < 1e-8
    th = torch.sqrt(torch.where(small, torch.ones_like(th2), th2))
    imag = torch.where(small, 0.5 - th2 / 48.0 + th2 * th2 / 3840.0, torch.sin(0.5 * th) / th)
    real = torch.where(small, 1.0 - th2 / 8.0 + th2 * th2 / 384.0, torch.cos(0.5 * th))
    q = torch.cat([imag * phi, real], -1)
    c1 = _cross(phi, tau)
    c2 = _cross(phi, c1)
    big = torch.sqrt(th2.clamp_min(0)) > 1e-4
    a = torch.where(big, (1 - torch.cos(th)) / (th * th), torch.zeros_like(th))
    b = torch.where(big, (th - torch.sin(th)) / (th * th * th), torch.zeros_like(th))
    t = tau + a * c1 + b * c2
    return torch.cat([t, q], -1)


def se3_mul(X, Y):
    return torch.cat([X[..., :3] + quat_rot(X[..., 3:], Y[..., :3]), quat_mul(X[..., 3:], Y[..., 3:])], -1)


def se3_inv(X):
    qi = X[..., 3:] * X.new_tensor([-1.0, -1.0, -1.0, 1.0])
    return torch.cat([-quat_rot(qi, X[..., :3]), qi], -1)


def se3_log(X):
    """(..., 7) -> (..., 6) [tau, phi] (unit quaternion assumed; theta away from 0 and pi)."""
    q = X[..., 3:]
    q = torch.where(q[..., 3:4] < 0, -q, q)
    v, w = q[..., :3], q[..., 3:4]
    n = torch.sqrt((v * v).sum(-1, keepdim=True) + 1e-300)
    phi = 2.0 * torch.atan2(n, w) / n * v
    th = torch.sqrt((phi * phi).sum(-1, keepdim=True) + 1e-300)
    coef = (1 - th * torch.cos(th / 2) / (2 * torch.sin(th / 2))) / (th * th)
    t = X[..., :3]
    c1 = _cross(phi, t)
    tau = t - 0.5 * c1 + coef * _cross(phi, c1)
    return torch.cat([tau, phi], -1)


# ---------------------------------------------------------------- Sim3 [t q s], tangent [tau phi sigma]

def sim3_mul(X, Y):
    t = X[..., :3] + X[..., 7:8] * quat_rot(X[..., 3:7], Y[..., :3])
    return torch.cat([t, quat_mul(X[..., 3:7], Y[..., 3:7]), X[..., 7:8] * Y[..., 7:8]], -1)


def sim3_inv(X):
    qi = X[..., 3:7] * X.new_tensor([-1.0, -1.0, -1.0, 1.0])
    si = 1.0 / X[..., 7:8]
    return torch.cat([-si * quat_rot(qi, X[..., :3]), qi, si], -1)


def _sim3_W(phi, sig):
    """3x3 W(phi, sigma) of the Sim3 exponential (translation = W tau), closed form with
    the small-angle / small-scale limits (the published Sim3 exponential used by lietorch)."""
    th = torch.linalg.norm(phi)
    Ph = torch.zeros(3, 3, dtype=phi.dtype)
    Ph[0, 1], Ph[0, 2], Ph[1, 0], Ph[1, 2], Ph[2, 0], Ph[2, 1] = -phi[2], phi[1], phi[2], -phi[0], -phi[1], phi[0]
    P2 = Ph @ Ph
    sc = torch.exp(sig)
    eps = 1e-6
    if abs(float(sig)) < eps:
        C = torch.ones((), dtype=phi.dtype)
        if float(th) < eps:
            A, B = 0.5 * C, C / 6.0
        else:
            A = (1 - torch.cos(th)) / (th * th)
            B = (th - torch.sin(th)) / th**3
    else:
        C = (sc - 1) / sig
        if float(th) < eps:
            s2 = sig * sig
            A = ((sig - 1) * sc + 1) / s2
            B = (sc * 0.5 * s2 + sc - 1 - sig * sc) / (s2 * sig)
        else:
            a = sc * torch.sin(th)
            b = sc * torch.cos(th)
            c = th * th + sig * sig
            A = (a * sig + (1 - b) * th) / (th * c)
            B = (C - ((b - 1) * sig + a * th) / c) / (th * th)
    return A * Ph + B * P2 + C * torch.eye(3, dtype=phi.dtype)


def sim3_exp(xi):
    """(P, 7) -> (P, 8)"""
    out = []
    for r in xi:
        q = se3_exp(torch.cat([torch.zeros(3, dtype=r.dtype), r[3:6]]))[3:]
        t = _sim3_W(r[3:6], r[6]) @ r[:3]
        out.append(torch.cat([t, q, torch.exp(r[6:7])]))
    return torch.stack(out)


def perturb(poses, eps):
    """Left tangent perturbation Exp(eps) * poses (eps (N, 6); eps = 0 gives poses)."""
    return se3_mul(se3_exp(eps), poses)


def _adj_t(tij, qij, X):
    """Ad(T)^T X for X (..., 6) [geom_kernels.cu:88-102]."""
    qi = qij * qij.new_tensor([-1.0, -1.0, -1.0, 1.0])
    a = quat_rot(qi, X[..., :3])
    b = quat_rot(qi, X[..., 3:]) + quat_rot(qi, _cross(X[..., :3], tij))
    return torch.cat([a, b], -1)


def ba_torch(poses, disps, intrinsics, disps_sens, targets, weights, eta, ii, jj, depth_active, t0, t1, iterations,
             lm, ep, alpha, detach_damping=True):
    """Returns (poses_out, disps_out, dx_last, dz_last); every input may carry autograd."""
    dt = torch.float64
    N, H, W = disps.shape
    HW = H * W
    E = ii.shape[0]
    P = t1 - t0
    ii_l, jj_l = [int(x) for x in ii], [int(x) for x in jj]
    kx = sorted(set(range(t0, t1)) | set(ii_l))
    K = len(kx)
    if eta.shape[0] != K:
        raise ValueError("eta rows != |kx|")
    row_of = {f: r for r, f in enumerate(kx)}
    fx, fy, cx, cy = intrinsics[0], intrinsics[1], intrinsics[2], intrinsics[3]
    vv, uu = torch.meshgrid(torch.arange(H, dtype=dt), torch.arange(W, dtype=dt), indexing="ij")
    uu, vv = uu.reshape(-1), vv.reshape(-1)
    act_f = depth_active.to(dt)
    poses = poses.to(dt)
    disps = disps.to(dt)
    sim3 = poses.shape[-1] == 8
    D = 7 if sim3 else 6
    dx = dz = None
    for _ in range(iterations):
        Bm = torch.zeros(D * P, D * P, dtype=dt)
        vb = torch.zeros(D * P, dtype=dt)
        Em = [torch.zeros(D * P, HW, dtype=dt) for _ in range(K)]
        Csum = [torch.zeros(HW, dtype=dt) for _ in range(K)]
        bsum = [torch.zeros(HW, dtype=dt) for _ in range(K)]
        for e in range(E):
            a, b = ii_l[e], jj_l[e]
            sij = torch.ones((), dtype=dt)
            if a == b:
                tij = torch.tensor([-0.1, 0.0, 0.0], dtype=dt)
                qij = torch.tensor([0.0, 0.0, 0.0, 1.0], dtype=dt)
            elif sim3:
                Tij = sim3_mul(poses[b], sim3_inv(poses[a]))
                tij, qij, sij = Tij[:3], Tij[3:7], Tij[7]
            else:
                Tij = se3_mul(poses[b], se3_inv(poses[a]))
                tij, qij = Tij[:3], Tij[3:]
            d = disps[a].reshape(-1)
            Xi = torch.stack([(uu - cx) / fx, (vv - cy) / fy, torch.ones_like(uu)], -1)
            Xj = sij * quat_rot(qij.expand(HW, 4), Xi) + d[:, None] * tij[None]
            x, y, z, h = Xj[:, 0], Xj[:, 1], Xj[:, 2], d
            ok = (z >= MIN_DEPTH).detach()
            zi = torch.where(ok, 1.0 / torch.where(ok, z, torch.ones_like(z)), torch.zeros_like(z))
            zi2 = zi * zi
            wu = torch.where(ok, 0.001 * weights[e, 0].reshape(-1).to(dt), torch.zeros_like(z))
            wv = torch.where(ok, 0.001 * weights[e, 1].reshape(-1).to(dt), torch.zeros_like(z))
            ru = targets[e, 0].reshape(-1).to(dt) - (fx * zi * x + cx)
            rv = targets[e, 1].reshape(-1).to(dt) - (fy * zi * y + cy)
            zero = torch.zeros_like(z)
            Jj_u = torch.stack([fx * h * zi, zero, -fx * x * h * zi2, -fx * x * y * zi2, fx * (1 + x * x * zi2),
                                -fx * y * zi], -1)
            Jj_v = torch.stack([zero, fy * h * zi, -fy * y * h * zi2, fy * (-1 - y * y * zi2), fy * x * y * zi2,
                                fy * x * zi], -1)
            Jz_u = fx * (tij[0] * zi - tij[2] * x * zi2)
            Jz_v = fy * (tij[1] * zi - tij[2] * y * zi2)
            if sim3:
                # target: tau d grad f, phi P x grad f, sigma 0; source: -d g, -(X3 x g), -X3.g, g = s R^T grad f
                qc = qij * qij.new_tensor([-1.0, -1.0, -1.0, 1.0])
                rows = []
                for gf in (torch.stack([fx * zi, zero, -fx * x * zi2], -1), torch.stack([zero, fy * zi, -fy * y * zi2], -1)):
                    g = sij * quat_rot(qc.expand(HW, 4), gf)
                    Ji = torch.cat([-h[:, None] * g, -torch.cross(Xi, g, dim=-1), -(Xi * g).sum(-1, keepdim=True)], -1)
                    Jj = torch.cat([h[:, None] * gf, torch.cross(Xj, gf, dim=-1), zero[:, None]], -1)
                    rows.append((Ji, Jj))
                (Ji_u, Jj_u), (Ji_v, Jj_v) = rows
            else:
                Ji_u = -_adj_t(tij.expand(HW, 3), qij.expand(HW, 4), Jj_u)
                Ji_v = -_adj_t(tij.expand(HW, 3), qij.expand(HW, 4), Jj_v)
            act = act_f[a]
            k = row_of[a]
            wpu, wpv = (wu * 0, wv * 0) if a == b else (wu, wv)
            slots = []
            if t0 <= a < t1:
                slots.append((a - t0, Ji_u, Ji_v))
            if t0 <= b < t1:
                slots.append((b - t0, Jj_u, Jj_v))
            for (pa, Ja_u, Ja_v) in slots:
                vb = vb.index_add(0, torch.arange(D * pa, D * pa + D),
                                  (wpu * ru)[:, None].mul(Ja_u).sum(0) + (wpv * rv)[:, None].mul(Ja_v).sum(0))
                for (pb, Jb_u, Jb_v) in slots:
                    blk = (Ja_u * wpu[:, None]).T @ Jb_u + (Ja_v * wpv[:, None]).T @ Jb_v
                    Bm = Bm.index_put((torch.arange(D * pa, D * pa + D)[:, None],
                                       torch.arange(D * pb, D * pb + D)[None, :]), blk, accumulate=True)
                Em[k] = Em[k].index_put((torch.arange(D * pa, D * pa + D),),
                                        act * (act * wu * Jz_u)[None, :] * Ja_u.T
                                        + act * (act * wv * Jz_v)[None, :] * Ja_v.T, accumulate=True)
            Csum[k] = Csum[k] + act * wu * Jz_u * Jz_u + act * wv * Jz_v * Jz_v
            bsum[k] = bsum[k] + act * wu * ru * Jz_u + act * wv * rv * Jz_v
        Cs, ws = [], []
        for k, f in enumerate(kx):
            act = act_f[f]
            dsens = disps_sens[f].reshape(-1).to(dt)
            msk = (dsens > 0).to(dt) * act
            Cs.append(act * (Csum[k] + eta[k].reshape(-1).to(dt) + msk * alpha) + (1 - act))
            dd = disps[f].reshape(-1) - dsens
            ws.append(act * (bsum[k] - msk * alpha * dd))
        Cc = torch.cat(Cs)
        wz = torch.cat(ws)
        Ef = torch.cat(Em, 1)
        Q = 1.0 / Cc
        S = Bm - (Ef * Q[None]) @ Ef.T
        yv = vb - Ef @ (Q * wz)
        dg = torch.diagonal(S)
        damp = ep + lm * (dg.detach() if detach_damping else dg)
        Sd = S + torch.diag(damp)
        dxi = torch.linalg.solve(Sd, yv)
        mask_rows = torch.ones(D * P, dtype=dt)
        mask_rows[:D] = 0.0  # pose t0's rows are left out of the back-substitution
        dzv = Q * (wz - Ef.T @ (dxi * mask_rows))
        dxf = dxi.view(P, D)
        newp = sim3_mul(sim3_exp(dxf), poses[t0:t1]) if sim3 else se3_mul(se3_exp(dxf), poses[t0:t1])
        poses = torch.cat([poses[:t0], newp, poses[t1:]], 0)
        dzr = dzv.view(K, H, W)
        idx = torch.tensor(kx)
        disps = disps.index_add(0, idx, dzr)
        dx, dz = dxf, dzr.reshape(K, HW)
    return poses, disps, dx, dz
