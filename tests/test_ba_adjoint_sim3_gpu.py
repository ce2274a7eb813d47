"""The hand-written BA adjoint of the Sim3 batched solve (group "sim3", poses (N, 8) [t q s],
tangent [tau phi sigma]; no counterpart in the reference, whose BA has neither Sim3 nor a
backward).

Two uneven Sim3 clips (12x16 depth maps, |i-j| <= 2 plus a loop pair, 2 LM iterations)
through vipe_b200.ba_autograd.bundle_adjust, a random-weighted smooth loss of the output poses
(as 8-vectors, differentiated along the left tangent) and depths, against torch autograd of the
dense FP64 Sim3 BA (oracle/ba_torch.py, the LM damping's dependence on diag(S) included):
relative error (norm over each gradient tensor) below 5e-4 for poses, depths, targets and
weights, and FP64 central differences (h = 1e-6) of the same torch BA on 16 random entries
below 1e-3.
"""

import numpy as np
import pytest
import torch

from oracle import ba_torch as bt
from vipe_b200 import ba_autograd as BA
from vipe_b200 import ba_batch as BB
from vipe_b200 import workloads as W

pytestmark = pytest.mark.gpu

ITERS, LM, EP, ALPHA = 2, 1e-4, 0.1, 0.001


def _batch():
    return W.make_ba_batch(2, seed=41, frames_range=(6, 7), radius=2, loops_mean=0.7, loop_gap=3, ht=12, wd=16,
                           intrinsics=(15.0, 15.0, 8.0, 6.0), outlier_frac=0.0, group="sim3")


def _weights(p, seed):
    g = np.random.default_rng(seed)
    N, H, W_ = p.disps.shape
    return torch.from_numpy(g.normal(size=(N, 8))), torch.from_numpy(g.normal(size=(N, H, W_)))


def _loss(poses, disps, cw):
    return (cw[0] * poses).sum() + (cw[1] * disps).sum()


def _torch_forward(p, eps, d0, tg, wt):
    return bt.ba_torch(bt.sim3_mul(bt.sim3_exp(eps), p.poses.double()), d0, p.intrinsics.double(),
                       p.disps_sens.double(), tg, wt, p.eta.double(), p.ii, p.jj, p.depth_active.double(), p.t0,
                       p.t1, ITERS, LM, EP, ALPHA, detach_damping=False)


def _torch_grads(p, cw):
    eps = torch.zeros(p.poses.shape[0], 7, dtype=torch.float64, requires_grad=True)
    d0 = p.disps.double().clone().requires_grad_(True)
    tg = p.targets.double().clone().requires_grad_(True)
    wt = p.weights.double().clone().requires_grad_(True)
    out = _torch_forward(p, eps, d0, tg, wt)
    _loss(out[0], out[1], cw).backward()
    return dict(poses=eps.grad.numpy(), disps=d0.grad.numpy(), targets=tg.grad.numpy(), weights=wt.grad.numpy())


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _cuda_grads(b, cws):
    plan = BB.BatchPlan(*b.sizes, b.ht, b.wd, "cuda", group="sim3", adjoint=True)
    t = {k: v.cuda() for k, v in b.tensors.items()}
    poses = t["poses"].clone().requires_grad_(True)
    disps = t["disps"].clone().requires_grad_(True)
    targets = t["targets"].clone().requires_grad_(True)
    weights = t["weights"].clone().requires_grad_(True)
    po, do = BA.bundle_adjust(plan, poses, disps, targets, weights, t["eta"], t["disps_sens"], t["intrinsics"],
                              t["ii"], t["jj"], t["depth_active"], ITERS, LM, EP, ALPHA)
    gpo, gdo = torch.zeros_like(po), torch.zeros_like(do)
    fo = 0
    for g in range(b.G):
        n = b.num_frames[g]
        zeta = torch.zeros(n, 7, dtype=torch.float64, requires_grad=True)
        pp = bt.sim3_mul(bt.sim3_exp(zeta), po[fo:fo + n].detach().cpu().double())
        (gz,) = torch.autograd.grad(_loss(pp, do[fo:fo + n].detach().cpu().double(), cws[g]), zeta)
        gpo[fo:fo + n, :7] = gz.float().cuda()
        gdo[fo:fo + n] = cws[g][1].float().cuda()
        fo += n
    torch.autograd.backward([po, do], [gpo, gdo])
    torch.cuda.synchronize()
    out, fo, eo = [], 0, 0
    for g in range(b.G):
        n, e = b.num_frames[g], b.num_edges[g]
        out.append(dict(poses=poses.grad[fo:fo + n, :7].double().cpu().numpy(),
                        disps=disps.grad[fo:fo + n].double().cpu().numpy(),
                        targets=targets.grad[eo:eo + e].double().cpu().numpy(),
                        weights=weights.grad[eo:eo + e].double().cpu().numpy()))
        fo, eo = fo + n, eo + e
    return out


def _fd(p, cw, name, idx, h=1e-6):
    vals = []
    for s in (h, -h):
        eps = torch.zeros(p.poses.shape[0], 7, dtype=torch.float64)
        d0, tg, wt = p.disps.double().clone(), p.targets.double().clone(), p.weights.double().clone()
        if name == "poses":
            eps[idx] = s
        else:
            {"disps": d0, "targets": tg, "weights": wt}[name][idx] += s
        with torch.no_grad():
            out = _torch_forward(p, eps, d0, tg, wt)
        vals.append(float(_loss(out[0], out[1], cw)))
    return (vals[0] - vals[1]) / (2 * h)


def test_sim3_adjoint_matches_torch_autograd_and_fd():
    b = _batch()
    clips = [b.clip(g) for g in range(b.G)]
    cws = [_weights(p, 60 + g) for g, p in enumerate(clips)]
    got = _cuda_grads(b, cws)
    for g, p in enumerate(clips):
        want = _torch_grads(p, cws[g])
        errs = {k: _rel(got[g][k], want[k]) for k in ("poses", "disps", "targets", "weights")}
        print(g, errs)
        assert all(v < 5e-4 for v in errs.values()), (g, errs)
    p, rng = clips[0], np.random.default_rng(5)
    N, H, W_ = p.disps.shape
    E = p.ii.shape[0]
    picks = []
    for _ in range(4):
        picks.append(("poses", (int(rng.integers(0, N)), int(rng.integers(0, 7)))))
        picks.append(("disps", (int(rng.integers(0, N)), int(rng.integers(0, H)), int(rng.integers(0, W_)))))
        picks.append(("targets", (int(rng.integers(0, E)), int(rng.integers(0, 2)), int(rng.integers(0, H)),
                                  int(rng.integers(0, W_)))))
        picks.append(("weights", (int(rng.integers(0, E)), int(rng.integers(0, 2)), int(rng.integers(0, H)),
                                  int(rng.integers(0, W_)))))
    gv = np.array([got[0][n][i] for n, i in picks])
    fd = np.array([_fd(p, cws[0], n, i) for n, i in picks])
    print("fd", _rel(gv, fd))
    assert _rel(gv, fd) < 1e-3


def test_sim3_differentiable_forward_equals_plain_solve():
    b = _batch()
    t = {k: v.cuda() for k, v in b.tensors.items()}
    plan = BB.BatchPlan(*b.sizes, b.ht, b.wd, "cuda", group="sim3", adjoint=True)
    po, do = BA.bundle_adjust(plan, t["poses"], t["disps"], t["targets"], t["weights"], t["eta"], t["disps_sens"],
                              t["intrinsics"], t["ii"], t["jj"], t["depth_active"], ITERS, LM, EP, ALPHA)
    plain = {k: v.clone() for k, v in t.items()}
    BB.BatchPlan(*b.sizes, b.ht, b.wd, "cuda", group="sim3").solve(**plain, iterations=ITERS, lm=LM, ep=EP,
                                                                     alpha=ALPHA)
    assert torch.equal(po, plain["poses"]) and torch.equal(do, plain["disps"])
