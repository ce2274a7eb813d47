"""Seeded synthetic inputs for the bundle-adjustment and correlation workloads.

No dataset is involved anywhere: every input is generated from a seed with the
shapes and value distributions the workloads are specified with.

BA generative model (all sizes in depth-map pixels):
  * SE3 trajectory: a random walk T_{i+1} = Exp([dt, dphi]) T_i with per-frame
    axis-angle steps dphi ~ N(0, 0.02^2) rad and translation steps dt ~ N(0, 0.05^2)
    per axis; poses are world-to-camera [tx ty tz qx qy qz qw] as in the
    reference's GraphBuffer;
  * ground-truth inverse depth: N(0,1) noise blurred with a Gaussian of sigma 4 px,
    min-max mapped to [0.1, 1.0];
  * targets: the ground-truth reprojection of every pixel of frame ii into frame
    jj (pinhole, u = column, v = row) plus N(0, 0.5^2) px; weights ~ U(0.1, 1) on
    both channels;
  * initial state: poses Exp(delta) T_gt with delta per axis N(0, (0.01/sqrt3)^2)
    rad and N(0, (0.02/sqrt3)^2) translation; disps d_gt * (1 + N(0, 0.05^2));
  * eta = 0.2 * U(1e-4, 1e-2) + 1e-7 per pixel (the range of the update
    operator's 0.01*softplus damping), disps_sens = 0, depth_active = 1.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch


# ---------------------------------------------------------------- SE3 helpers (float64, numpy)

def _quat_mul(a, b):
    ax, ay, az, aw = a[..., 0], a[..., 1], a[..., 2], a[..., 3]
    bx, by, bz, bw = b[..., 0], b[..., 1], b[..., 2], b[..., 3]
    return np.stack(
        [
            aw * bx + ax * bw + ay * bz - az * by,
            aw * by - ax * bz + ay * bw + az * bx,
            aw * bz + ax * by - ay * bx + az * bw,
            aw * bw - ax * bx - ay * by - az * bz,
        ],
        -1,
    )


def _quat_rot(q, x):
    v = q[..., :3]
    w = q[..., 3:4]
    uv = 2.0 * np.cross(v, x)
    return x + w * uv + np.cross(v, uv)


def se3_exp(xi):
    """xi (..., 6) = [tau, phi] -> (..., 7) [t, q] (exact series-free form)."""
    tau, phi = xi[..., :3], xi[..., 3:]
    th = np.linalg.norm(phi, axis=-1, keepdims=True)
    small = th < 1e-8
    ths = np.where(small, 1.0, th)
    imag = np.where(small, 0.5, np.sin(0.5 * ths) / ths)
    q = np.concatenate([imag * phi, np.cos(0.5 * th)], -1)
    A = np.where(small, 0.5, (1 - np.cos(ths)) / ths**2)
    B = np.where(small, 1.0 / 6.0, (ths - np.sin(ths)) / ths**3)
    c1 = np.cross(phi, tau)
    c2 = np.cross(phi, c1)
    t = tau + A * c1 + B * c2
    return np.concatenate([t, q], -1)


def se3_mul(X, Y):
    t = X[..., :3] + _quat_rot(X[..., 3:], Y[..., :3])
    return np.concatenate([t, _quat_mul(X[..., 3:], Y[..., 3:])], -1)


def se3_inv(X):
    qi = X[..., 3:] * np.array([-1, -1, -1, 1.0])
    return np.concatenate([-_quat_rot(qi, X[..., :3]), qi], -1)


def sim3_mul(X, Y):
    """(..., 8) Sim3 [t q s] composition X * Y = (tX + sX R_X tY, qX qY, sX sY)."""
    t = X[..., :3] + X[..., 7:8] * _quat_rot(X[..., 3:7], Y[..., :3])
    return np.concatenate([t, _quat_mul(X[..., 3:7], Y[..., 3:7]), X[..., 7:8] * Y[..., 7:8]], -1)


def se3_log(X):
    """(..., 7) -> (..., 6) [tau, phi]."""
    q = X[..., 3:] / np.linalg.norm(X[..., 3:], axis=-1, keepdims=True)
    q = np.where(q[..., 3:4] < 0, -q, q)
    v, w = q[..., :3], q[..., 3:4]
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    small = n < 1e-10
    ns = np.where(small, 1.0, n)
    fac = np.where(small, 2.0 / w, 2.0 * np.arctan2(ns, w) / ns)
    phi = fac * v
    th = np.linalg.norm(phi, axis=-1, keepdims=True)
    ths = np.where(th < 1e-8, 1.0, th)
    coef = np.where(th < 1e-8, 1.0 / 12.0, (1 - ths * np.cos(ths / 2) / (2 * np.sin(ths / 2))) / ths**2)
    t = X[..., :3]
    c1 = np.cross(phi, t)
    c2 = np.cross(phi, c1)
    tau = t - 0.5 * c1 + coef * c2
    return np.concatenate([tau, phi], -1)


# ---------------------------------------------------------------- BA workload

@dataclass
class BAProblem:
    """Inputs of one dense BA solve in the reference's slam_ext layouts (CPU tensors)."""

    poses: torch.Tensor  # (N, 7) f32
    disps: torch.Tensor  # (N, H, W) f32
    intrinsics: torch.Tensor  # (4,) f32
    disps_sens: torch.Tensor  # (N, H, W) f32
    targets: torch.Tensor  # (E, 2, H, W) f32
    weights: torch.Tensor  # (E, 2, H, W) f32
    eta: torch.Tensor  # (|kx|, H, W) f32
    ii: torch.Tensor  # (E,) int64
    jj: torch.Tensor  # (E,) int64
    depth_active: torch.Tensor  # (N,) f32
    t0: int
    t1: int
    iterations: int
    lm: float = 1e-4
    ep: float = 0.1
    alpha: float = 0.001
    poses_gt: torch.Tensor | None = None
    disps_gt: torch.Tensor | None = None

    def to(self, device) -> "BAProblem":
        kw = {}
        for k, v in self.__dict__.items():
            kw[k] = v.to(device) if isinstance(v, torch.Tensor) else v
        return BAProblem(**kw)

    def clone(self) -> "BAProblem":
        kw = {}
        for k, v in self.__dict__.items():
            kw[k] = v.clone() if isinstance(v, torch.Tensor) else v
        return BAProblem(**kw)

    @property
    def num_edges(self) -> int:
        return int(self.ii.shape[0])


def _gaussian_blur(x: np.ndarray, sigma: float) -> np.ndarray:
    r = int(math.ceil(3 * sigma))
    g = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    g /= g.sum()
    t = torch.from_numpy(x)[:, None]
    kx = torch.from_numpy(g).view(1, 1, 1, -1)
    ky = torch.from_numpy(g).view(1, 1, -1, 1)
    t = torch.nn.functional.pad(t, (r, r, 0, 0), mode="replicate")
    t = torch.nn.functional.conv2d(t, kx)
    t = torch.nn.functional.pad(t, (0, 0, r, r), mode="replicate")
    t = torch.nn.functional.conv2d(t, ky)
    return t[:, 0].numpy()


def band_edges(n: int, radius: int) -> list[tuple[int, int]]:
    """All ordered pairs (i, j) with 0 < |i - j| <= radius, i-major order."""
    return [(i, j) for i in range(n) for j in range(n) if i != j and abs(i - j) <= radius]


def random_long_edges(n: int, count: int, min_gap: int, rng: np.random.Generator) -> list[tuple[int, int]]:
    """`count` distinct unordered pairs with |i - j| > min_gap, both directions."""
    pairs: set[tuple[int, int]] = set()
    out = []
    guard = 0
    while len(pairs) < count and guard < 100000:
        guard += 1
        i, j = sorted(rng.integers(0, n, size=2).tolist())
        if j - i > min_gap and (i, j) not in pairs:
            pairs.add((i, j))
            out += [(i, j), (j, i)]
    return out


def make_ba_problem(
    n_frames: int,
    edges: list[tuple[int, int]],
    seed: int,
    ht: int = 48,
    wd: int = 64,
    t0: int = 2,
    iterations: int = 2,
    intrinsics=(60.0, 60.0, 32.0, 24.0),
) -> BAProblem:
    rng = np.random.default_rng(seed)
    # trajectory
    T = np.zeros((n_frames, 7))
    T[0] = [0, 0, 0, 0, 0, 0, 1]
    for i in range(1, n_frames):
        step = np.concatenate([rng.normal(0, 0.05, 3), rng.normal(0, 0.02, 3)])
        T[i] = se3_mul(se3_exp(step), T[i - 1])
    # depth
    noise = rng.normal(0, 1, (n_frames, ht, wd))
    sm = _gaussian_blur(noise, 4.0)
    lo = sm.reshape(n_frames, -1).min(1)[:, None, None]
    hi = sm.reshape(n_frames, -1).max(1)[:, None, None]
    d_gt = 0.1 + 0.9 * (sm - lo) / np.maximum(hi - lo, 1e-12)
    fx, fy, cx, cy = intrinsics
    vv, uu = np.meshgrid(np.arange(ht, dtype=np.float64), np.arange(wd, dtype=np.float64), indexing="ij")
    ii = np.array([e[0] for e in edges], dtype=np.int64)
    jj = np.array([e[1] for e in edges], dtype=np.int64)
    E = len(edges)
    targets = np.zeros((E, 2, ht, wd))
    for k, (i, j) in enumerate(edges):
        X = np.stack([(uu - cx) / fx, (vv - cy) / fy, np.ones_like(uu)], -1)
        Tij = se3_mul(T[j], se3_inv(T[i]))
        Xj = _quat_rot(Tij[3:], X) + d_gt[i][..., None] * Tij[:3]
        z = Xj[..., 2]
        targets[k, 0] = fx * Xj[..., 0] / z + cx
        targets[k, 1] = fy * Xj[..., 1] / z + cy
    targets += rng.normal(0, 0.5, targets.shape)
    weights = rng.uniform(0.1, 1.0, (E, 2, ht, wd))
    # initial state
    P0 = T.copy()
    for i in range(n_frames):
        delta = np.concatenate([rng.normal(0, 0.02 / math.sqrt(3), 3), rng.normal(0, 0.01 / math.sqrt(3), 3)])
        P0[i] = se3_mul(se3_exp(delta), T[i])
    d0 = d_gt * (1 + rng.normal(0, 0.05, d_gt.shape))
    t1 = n_frames
    kx = np.unique(np.concatenate([np.arange(t0, t1), ii]))
    eta = 0.2 * rng.uniform(1e-4, 1e-2, (len(kx), ht, wd)) + 1e-7
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a)).float()
    return BAProblem(
        poses=f32(P0),
        disps=f32(d0),
        intrinsics=torch.tensor(intrinsics, dtype=torch.float32),
        disps_sens=torch.zeros(n_frames, ht, wd),
        targets=f32(targets),
        weights=f32(weights),
        eta=f32(eta),
        ii=torch.from_numpy(ii),
        jj=torch.from_numpy(jj),
        depth_active=torch.ones(n_frames),
        t0=t0,
        t1=t1,
        iterations=iterations,
        poses_gt=f32(T),
        disps_gt=f32(d_gt),
    )


def ba_config0() -> BAProblem:
    """8 keyframes, |i-j| <= 2 (26 edges), 2 LM iterations, first 2 poses fixed."""
    return make_ba_problem(8, band_edges(8, 2), seed=1000, t0=2, iterations=2)


def ba_config1() -> BAProblem:
    """64 keyframes, |i-j| <= 3 plus 128 random long-range pairs (628 edges), 4 iterations."""
    rng = np.random.default_rng(1001)
    edges = band_edges(64, 3) + random_long_edges(64, 128, 8, rng)
    return make_ba_problem(64, edges, seed=1001, t0=2, iterations=4)


def ba_backend(n_frames: int = 256, hub_every: int = 16, hub_degree: int = 40, ht: int = 48, wd: int = 64,
               seed: int = 1005, iterations: int = 2, t0: int = 1) -> BAProblem:
    """A backend-style global BA window: every keyframe in [t0, n_frames) optimised,
    edges |i-j| <= 3 plus, from every `hub_every`-th keyframe, `hub_degree` loop pairs
    (|i-j| > 8, both directions) to random keyframes, so the hubs' depth frames are
    coupled to hub_degree + 7 window poses (the shape proximity and loop-closure factors
    give ViPE's backend, vipe/slam/components/factor_graph.py:376-486)."""
    rng = np.random.default_rng(seed)
    edges = band_edges(n_frames, 3)
    have = set(edges)
    for h in range(0, n_frames, hub_every):
        far = [j for j in range(n_frames) if abs(j - h) > 8]
        for j in rng.choice(far, size=min(hub_degree, len(far)), replace=False).tolist():
            for e in ((h, j), (j, h)):
                if e not in have:
                    have.add(e)
                    edges.append(e)
    scale = wd / 64.0
    return make_ba_problem(n_frames, edges, seed=seed, ht=ht, wd=wd, t0=t0, iterations=iterations,
                           intrinsics=(60.0 * scale, 60.0 * scale, wd / 2.0, ht / 2.0))


def frame_slots(p: BAProblem) -> np.ndarray:
    """Window poses coupled to each depth frame of `p` (its own pose, if in the window, and the
    distinct in-window targets of its edges), in the order of the sorted depth frames."""
    ii, jj = p.ii.numpy(), p.jj.numpy()
    kx = np.unique(np.concatenate([np.arange(p.t0, p.t1), ii]))
    out = []
    for k in kx:
        s = {int(j) for j in jj[ii == k] if p.t0 <= j < p.t1}
        if p.t0 <= k < p.t1:
            s.add(int(k))
        out.append(len(s))
    return np.array(out)


def ba_small(n_frames: int = 6, ht: int = 12, wd: int = 16, radius: int = 2, seed: int = 7, iterations: int = 2,
             t0: int = 1) -> BAProblem:
    """A reduced-size problem with the same generative model (fast CPU oracle cases)."""
    return make_ba_problem(n_frames, band_edges(n_frames, radius), seed=seed, ht=ht, wd=wd, t0=t0,
                           iterations=iterations, intrinsics=(15.0, 15.0, wd / 2.0, ht / 2.0))


# ---------------------------------------------------------------- batched workload (many uneven clips)

def _torch_quat_rot(q, x):
    v, w = q[..., :3], q[..., 3:4]
    uv = 2.0 * torch.cross(v, x, dim=-1)
    return x + w * uv + torch.cross(v, uv, dim=-1)


def _torch_quat_mul(a, b):
    ax, ay, az, aw = a.unbind(-1)
    bx, by, bz, bw = b.unbind(-1)
    return torch.stack([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                        aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz], -1)


def _torch_relative(Ti, Tj):
    """Tij = Tj * Ti^-1 for (..., 7) SE3 or (..., 8) Sim3 poses."""
    qi_inv = Ti[..., 3:7] * Ti.new_tensor([-1.0, -1.0, -1.0, 1.0])
    if Ti.shape[-1] == 8:
        si_inv = 1.0 / Ti[..., 7:8]
        ti_inv = -si_inv * _torch_quat_rot(qi_inv, Ti[..., :3])
        q = _torch_quat_mul(Tj[..., 3:7], qi_inv)
        t = Tj[..., :3] + Tj[..., 7:8] * _torch_quat_rot(Tj[..., 3:7], ti_inv)
        return torch.cat([t, q, Tj[..., 7:8] * si_inv], -1)
    ti_inv = -_torch_quat_rot(qi_inv, Ti[..., :3])
    q = _torch_quat_mul(Tj[..., 3:], qi_inv)
    t = Tj[..., :3] + _torch_quat_rot(Tj[..., 3:], ti_inv)
    return torch.cat([t, q], -1)


@dataclass
class BABatch:
    """Concatenated inputs of many clips (the BatchPlan layout) plus per-clip sizes."""

    tensors: dict  # BATCH_KEYS -> tensor on `device`
    num_frames: list
    num_edges: list
    num_kx: list
    t0: list
    t1: list
    ht: int
    wd: int
    poses_gt: torch.Tensor
    disps_gt: torch.Tensor

    @property
    def sizes(self):
        return (self.num_frames, self.num_edges, self.num_kx, self.t0, self.t1)

    @property
    def G(self) -> int:
        return len(self.num_frames)

    def clip(self, g: int) -> BAProblem:
        """Clip g as a standalone BAProblem (CPU tensors), for per-graph reference solves."""
        fo, eo, ko = (sum(x[:g]) for x in (self.num_frames, self.num_edges, self.num_kx))
        n, e, k = self.num_frames[g], self.num_edges[g], self.num_kx[g]
        t = self.tensors
        # slice on the batch's device, then copy only the clip to the host
        return BAProblem(poses=t["poses"][fo:fo + n].cpu(), disps=t["disps"][fo:fo + n].cpu(),
                         intrinsics=t["intrinsics"][g].cpu(), disps_sens=t["disps_sens"][fo:fo + n].cpu(),
                         targets=t["targets"][eo:eo + e].cpu(), weights=t["weights"][eo:eo + e].cpu(),
                         eta=t["eta"][ko:ko + k].cpu(), ii=t["ii"][eo:eo + e].cpu(), jj=t["jj"][eo:eo + e].cpu(),
                         depth_active=t["depth_active"][fo:fo + n].cpu(), t0=self.t0[g], t1=self.t1[g],
                         iterations=4, poses_gt=self.poses_gt[fo:fo + n].cpu(), disps_gt=self.disps_gt[fo:fo + n].cpu())


def make_ba_batch(num_clips: int, seed: int, frames_range=(8, 96), radius: int = 3, loops_mean: float = 4.0,
                  loop_gap: int = 8, outlier_frac: float = 0.01, ht: int = 48, wd: int = 64, t0: int = 2,
                  intrinsics=(60.0, 60.0, 32.0, 24.0), device="cpu", group: str = "se3") -> BABatch:
    """Many clips of the BA generative model with uneven sizes.

    Keyframe counts ~ U{frames_range}; edges |i-j| <= radius plus Poisson(loops_mean)
    random loop pairs with |i-j| > loop_gap (both directions); a fraction
    `outlier_frac` of target entries is replaced by U(-20, 20) px with weight
    0.05.  Structure comes from numpy (seeded), the bulk noise from a seeded
    torch generator on `device` (generation runs on the GPU for large batches).
    group="sim3": poses are Sim3 [t q s]; each trajectory step also scales by
    exp(N(0, 0.02^2)) and the initial poses by exp(N(0, 0.01^2)).
    """
    sim3 = group == "sim3"
    rng = np.random.default_rng(seed)
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    nf = rng.integers(frames_range[0], frames_range[1] + 1, size=num_clips).tolist()
    ii_l, jj_l, ne, nk = [], [], [], []
    T_all = []
    for g in range(num_clips):
        n = nf[g]
        edges = band_edges(n, radius)
        nl = int(rng.poisson(loops_mean))
        if n - 1 > loop_gap and nl > 0:
            edges += random_long_edges(n, nl, loop_gap, rng)
        ii_l += [e[0] for e in edges]
        jj_l += [e[1] for e in edges]
        ne.append(len(edges))
        kx = np.unique(np.concatenate([np.arange(t0, n), np.array([e[0] for e in edges], dtype=np.int64)]))
        nk.append(len(kx))
        T = np.zeros((n, 7))
        T[0] = [0, 0, 0, 0, 0, 0, 1]
        steps = np.concatenate([rng.normal(0, 0.05, (n, 3)), rng.normal(0, 0.02, (n, 3))], 1)
        if sim3:
            T = np.concatenate([T, np.ones((n, 1))], 1)
            sc = np.exp(rng.normal(0, 0.02, n))
            for i in range(1, n):
                T[i] = sim3_mul(np.concatenate([se3_exp(steps[i]), [sc[i]]]), T[i - 1])
        else:
            for i in range(1, n):
                T[i] = se3_mul(se3_exp(steps[i]), T[i - 1])
        T_all.append(T)
    Nt, Et, Kt = sum(nf), sum(ne), sum(nk)
    T_gt = torch.from_numpy(np.concatenate(T_all)).to(dev)
    frame_off = np.concatenate([[0], np.cumsum(nf)[:-1]])
    clip_of_edge = np.repeat(np.arange(num_clips), ne)
    ii = torch.tensor(ii_l, dtype=torch.int64, device=dev)
    jj = torch.tensor(jj_l, dtype=torch.int64, device=dev)
    gi = ii + torch.from_numpy(frame_off[clip_of_edge]).to(dev)
    gj = jj + torch.from_numpy(frame_off[clip_of_edge]).to(dev)
    # ground-truth inverse depth: blurred noise mapped to [0.1, 1]
    noise = torch.randn(Nt, 1, ht, wd, generator=gen, device=dev, dtype=torch.float64)
    r = 12
    k1 = torch.exp(-0.5 * (torch.arange(-r, r + 1, device=dev, dtype=torch.float64) / 4.0) ** 2)
    k1 = k1 / k1.sum()
    sm = torch.nn.functional.conv2d(torch.nn.functional.pad(noise, (r, r, 0, 0), mode="replicate"), k1.view(1, 1, 1, -1))
    sm = torch.nn.functional.conv2d(torch.nn.functional.pad(sm, (0, 0, r, r), mode="replicate"), k1.view(1, 1, -1, 1))
    sm = sm[:, 0]
    lo = sm.flatten(1).min(1).values.view(-1, 1, 1)
    hi = sm.flatten(1).max(1).values.view(-1, 1, 1)
    d_gt = 0.1 + 0.9 * (sm - lo) / (hi - lo).clamp_min(1e-12)
    fx, fy, cx, cy = intrinsics
    vv, uu = torch.meshgrid(torch.arange(ht, device=dev, dtype=torch.float64),
                            torch.arange(wd, device=dev, dtype=torch.float64), indexing="ij")
    X = torch.stack([(uu - cx) / fx, (vv - cy) / fy, torch.ones_like(uu)], -1)  # (H, W, 3)
    targets = torch.empty(Et, 2, ht, wd, device=dev, dtype=torch.float32)
    weights = torch.empty(Et, 2, ht, wd, device=dev, dtype=torch.float32)
    chunk = 4096
    for e0 in range(0, Et, chunk):
        e1 = min(Et, e0 + chunk)
        Tij = _torch_relative(T_gt[gi[e0:e1]], T_gt[gj[e0:e1]])  # (c, 7) or (c, 8)
        RX = _torch_quat_rot(Tij[:, None, None, 3:7], X[None])
        if sim3:
            RX = RX * Tij[:, None, None, 7:8]
        Xj = RX + d_gt[gi[e0:e1]][..., None] * Tij[:, None, None, :3]
        z = Xj[..., 2]
        tg = torch.stack([fx * Xj[..., 0] / z + cx, fy * Xj[..., 1] / z + cy], 1)
        tg = tg + 0.5 * torch.randn(tg.shape, generator=gen, device=dev, dtype=torch.float64)
        wt = torch.rand(tg.shape, generator=gen, device=dev, dtype=torch.float64) * 0.9 + 0.1
        if outlier_frac > 0:
            out = torch.rand(tg.shape, generator=gen, device=dev, dtype=torch.float64) < outlier_frac
            tg = torch.where(out, torch.rand(tg.shape, generator=gen, device=dev, dtype=torch.float64) * 40 - 20, tg)
            wt = torch.where(out, torch.full_like(wt, 0.05), wt)
        targets[e0:e1] = tg.float()
        weights[e0:e1] = wt.float()
    # initial state
    delta = torch.cat([torch.randn(Nt, 3, generator=gen, device=dev, dtype=torch.float64) * (0.02 / math.sqrt(3)),
                       torch.randn(Nt, 3, generator=gen, device=dev, dtype=torch.float64) * (0.01 / math.sqrt(3))], 1)
    if sim3:
        ds = torch.exp(0.01 * torch.randn(Nt, 1, generator=gen, device=dev, dtype=torch.float64))
        dl = np.concatenate([se3_exp(delta.cpu().numpy()), ds.cpu().numpy()], 1)
        P0 = torch.from_numpy(sim3_mul(dl, T_gt.cpu().numpy())).to(dev)
    else:
        P0 = torch.from_numpy(se3_mul(se3_exp(delta.cpu().numpy()), T_gt.cpu().numpy())).to(dev)
    d0 = d_gt * (1 + 0.05 * torch.randn(d_gt.shape, generator=gen, device=dev, dtype=torch.float64))
    eta = 0.2 * (torch.rand(Kt, ht, wd, generator=gen, device=dev, dtype=torch.float64) * (1e-2 - 1e-4) + 1e-4) + 1e-7
    tensors = dict(
        poses=P0.float().contiguous(), disps=d0.float().contiguous(),
        intrinsics=torch.tensor(intrinsics, dtype=torch.float32, device=dev).repeat(num_clips, 1).contiguous(),
        disps_sens=torch.zeros(Nt, ht, wd, device=dev), targets=targets, weights=weights,
        eta=eta.float().contiguous(), ii=ii, jj=jj, depth_active=torch.ones(Nt, device=dev),
    )
    return BABatch(tensors=tensors, num_frames=nf, num_edges=ne, num_kx=nk, t0=[t0] * num_clips, t1=nf, ht=ht, wd=wd,
                   poses_gt=T_gt.float(), disps_gt=d_gt.float())


def ba_config4_se3(device="cpu", num_clips: int = 256) -> BABatch:
    """256 clips, keyframes ~ U{8..96}, |i-j| <= 3 + Poisson(4) loops, 1% outliers (SE3 form)."""
    return make_ba_batch(num_clips, seed=1004, device=device)


def ba_config4(device="cpu", num_clips: int = 256) -> BABatch:
    """256 clips, keyframes ~ U{8..96}, |i-j| <= 3 + Poisson(4) loops, 1% outliers, Sim3 poses."""
    return make_ba_batch(num_clips, seed=1004, device=device, group="sim3")
