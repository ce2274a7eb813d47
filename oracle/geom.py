"""FP64 numpy restatement of slam_ext's geometry helpers — TEST INFRASTRUCTURE ONLY.

Follows vipe csrc/slam_ext/geom_kernels.cu: projmap :526-611, frame_distance
:613-768, depth_filter :770-885, iproj :887-953 (pinhole, MIN_DEPTH 0.25).
"""

from __future__ import annotations

import numpy as np

from .lie import qmat, qmul

MIN_DEPTH = 0.25


def _rel(Ti, Tj):
    qi, qj = Ti[3:], Tj[3:]
    qij = qmul(qj, qi * np.array([-1, -1, -1, 1.0]))
    tij = Tj[:3] - qmat(qij) @ Ti[:3]
    return tij, qij


def _grid(ht, wd):
    v, u = np.meshgrid(np.arange(ht, dtype=np.float64), np.arange(wd, dtype=np.float64), indexing="ij")
    return u, v


def _act(t, q, X):
    R = qmat(q)
    P = np.einsum("ij,hwj->hwi", R, X[..., :3]) + X[..., 3:4] * t
    return np.concatenate([P, X[..., 3:4]], -1)


def projmap(poses, disps, intr, ii, jj):
    poses, disps = np.asarray(poses, np.float64), np.asarray(disps, np.float64)
    fx, fy, cx, cy = np.asarray(intr, np.float64)[:4]
    E = len(ii)
    _, H, W = disps.shape
    u, v = _grid(H, W)
    coords = np.zeros((E, H, W, 3))
    valid = np.zeros((E, H, W, 1))
    for e, (a, b) in enumerate(zip(ii, jj)):
        tij, qij = _rel(poses[a], poses[b])
        X = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u), disps[a]], -1)
        Xj = _act(tij, qij, X)
        z = Xj[..., 2]
        ok = z > 0.01
        coords[e, ..., 0] = np.where(ok, fx * Xj[..., 0] / np.where(ok, z, 1) + cx, u)
        coords[e, ..., 1] = np.where(ok, fy * Xj[..., 1] / np.where(ok, z, 1) + cy, v)
        valid[e, ..., 0] = (z > MIN_DEPTH).astype(np.float64)
    return coords, valid


def frame_distance(poses, disps, intr, pi, pj, qi, qj, di, beta):
    poses, disps = np.asarray(poses, np.float64), np.asarray(disps, np.float64)
    intr = np.asarray(intr, np.float64).reshape(-1, 4)
    _, H, W = disps.shape
    u, v = _grid(H, W)
    out = np.zeros(len(pi))
    for k in range(len(pi)):
        fxi, fyi, cxi, cyi = intr[qi[k]]
        fxj, fyj, cxj, cyj = intr[qj[k]]
        tij, qij = _rel(poses[pi[k]], poses[pj[k]])
        d = disps[di[k]]
        X = np.stack([(u - cxi) / fxi, (v - cyi) / fyi, np.ones_like(u), d], -1)
        Xj = _act(tij, qij, X)
        du = fxj * Xj[..., 0] / Xj[..., 2] + cxj - u
        dv = fyj * Xj[..., 1] / Xj[..., 2] + cyj - v
        full = np.sqrt(du * du + dv * dv)
        okf = Xj[..., 2] > MIN_DEPTH
        Xt = X[..., :3] + d[..., None] * tij
        du = fxj * Xt[..., 0] / Xt[..., 2] + cxj - u
        dv = fyj * Xt[..., 1] / Xt[..., 2] + cyj - v
        trans = np.sqrt(du * du + dv * dv)
        okt = Xt[..., 2] > MIN_DEPTH
        acc = (beta * full * okf).sum() + ((1 - beta) * trans * okt).sum()
        valid = beta * okf.sum() + (1 - beta) * okt.sum()
        total = H * W * (beta + (1 - beta))
        out[k] = 1000.0 if valid / (total + 1e-8) < 0.75 else acc / valid
    return out


def iproj(poses, disps, intr):
    poses, disps = np.asarray(poses, np.float64), np.asarray(disps, np.float64)
    fx, fy, cx, cy = np.asarray(intr, np.float64)[:4]
    N, H, W = disps.shape
    u, v = _grid(H, W)
    out = np.zeros((N, H, W, 3))
    for b in range(N):
        X = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u), disps[b]], -1)
        Xj = _act(poses[b, :3], poses[b, 3:], X)
        out[b] = Xj[..., :3] / Xj[..., 3:4]
    return out


def depth_filter(poses, disps, intr, ix, thresh):
    poses, disps = np.asarray(poses, np.float64), np.asarray(disps, np.float64)
    fx, fy, cx, cy = np.asarray(intr, np.float64)[:4]
    N, H, W = disps.shape
    u, v = _grid(H, W)
    out = np.zeros((len(ix), H, W))
    for k, i in enumerate(ix):
        for nb in range(6):
            j = i - nb - 1 if nb < 3 else i + nb - 2
            if j < 0 or j >= N:
                continue
            tij, qij = _rel(poses[i], poses[j])
            X = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u), disps[i]], -1)
            Xj = _act(tij, qij, X)
            uj = fx * Xj[..., 0] / Xj[..., 2] + cx
            vj = fy * Xj[..., 1] / Xj[..., 2] + cy
            dj = Xj[..., 3] / Xj[..., 2]
            u0, v0 = np.floor(uj).astype(int), np.floor(vj).astype(int)
            ok = (u0 >= 0) & (v0 >= 0) & (u0 < W - 1) & (v0 < H - 1)
            u0c, v0c = np.clip(u0, 0, W - 2), np.clip(v0, 0, H - 2)
            t = thresh[k]
            hit = np.zeros_like(ok)
            for dy in (0, 1):
                for dx in (0, 1):
                    hit |= np.abs(1.0 / dj - 1.0 / disps[j][v0c + dy, u0c + dx]) < t
            out[k] += (ok & hit).astype(np.float64)
    return out
