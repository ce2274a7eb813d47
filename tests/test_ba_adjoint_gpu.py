"""The hand-written BA adjoint on the GPU (vipe_b200.ba_autograd).

Compared, for a random-weighted loss of pose log-errors and depth errors, with
  * torch autograd of the dense FP64 torch BA, the LM damping's dependence on
    diag(S) differentiated too (the same mathematics): relative error (norm
    over each gradient tensor) below 2e-4 for poses, depths, targets and weights;
  * FP64 central finite differences (h = 1e-6) of the C++ oracle on 32 random
    entries of targets, weights, initial poses (left tangent) and initial
    depths: relative error (norm over the 32 entries) below 1e-3.
Cases: a small graph with a stereo edge and an inactive depth frame, and the
training window of 4 clips x 7 frames at 48x64 (|i-j| <= 2, 2 LM iterations).
"""

import numpy as np
import pytest
import torch

import oracle.ba as ob
from oracle import ba_torch as bt
from vipe_b200 import ba_autograd as BA
from vipe_b200 import ba_batch as BB
from vipe_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _small_problem():
    p = W.ba_small(n_frames=6, ht=12, wd=16, radius=2, seed=5, iterations=2, t0=2)
    p.ii = torch.cat([p.ii, torch.tensor([3])])
    p.jj = torch.cat([p.jj, torch.tensor([3])])
    p.targets = torch.cat([p.targets, p.targets[:1] + 0.3], 0)
    p.weights = torch.cat([p.weights, p.weights[:1]], 0)
    p.depth_active[4] = 0.0
    return p


def _window_problems():
    out = []
    for c in range(4):
        p = W.make_ba_problem(7, W.band_edges(7, 2), seed=3000 + c, t0=2, iterations=2)
        out.append(p)
    return out


def _loss_weights(p, seed):
    g = np.random.default_rng(seed)
    N, H, W_ = p.disps.shape
    return g.normal(size=(N, 6)), g.normal(size=(N, H, W_))


def _loss_torch(poses, disps, p, cw):
    cp, cd = (torch.from_numpy(x) for x in cw)
    gt = p.poses_gt.double()
    err = bt.se3_log(bt.se3_mul(bt.se3_inv(gt), poses))
    return (cp * err).sum() + (cd * (disps - p.disps_gt.double())).sum()


def _torch_grads(p, cw):
    eps = torch.zeros(p.poses.shape[0], 6, dtype=torch.float64, requires_grad=True)
    d0 = p.disps.double().clone().requires_grad_(True)
    tg = p.targets.double().clone().requires_grad_(True)
    wt = p.weights.double().clone().requires_grad_(True)
    out = bt.ba_torch(bt.perturb(p.poses.double(), eps), d0, p.intrinsics.double(), p.disps_sens.double(), tg, wt,
                      p.eta.double(), p.ii, p.jj, p.depth_active.double(), p.t0, p.t1, p.iterations, p.lm, p.ep,
                      p.alpha, detach_damping=False)
    _loss_torch(out[0], out[1], p, cw).backward()
    return dict(poses=eps.grad.numpy(), disps=d0.grad.numpy(), targets=tg.grad.numpy(), weights=wt.grad.numpy())


def _cuda_grads(problems, cws):
    """Runs the batched forward + adjoint on `problems`; returns per-problem gradient dicts."""
    plan = BB.BatchPlan.for_problems(problems, "cuda", adjoint=True)
    batch = BB.concat_problems(problems, device="cuda")
    poses = batch["poses"].clone().requires_grad_(True)
    disps = batch["disps"].clone().requires_grad_(True)
    targets = batch["targets"].clone().requires_grad_(True)
    weights = batch["weights"].clone().requires_grad_(True)
    it = problems[0].iterations
    po, do = BA.bundle_adjust(plan, poses, disps, targets, weights, batch["eta"], batch["disps_sens"],
                              batch["intrinsics"], batch["ii"], batch["jj"], batch["depth_active"], it,
                              problems[0].lm, problems[0].ep, problems[0].alpha)
    # incoming gradients: left-tangent for poses (lietorch layout), plain for disps
    gpo = torch.zeros_like(po)
    gdo = torch.zeros_like(do)
    fo = 0
    for p, cw in zip(problems, cws):
        n = p.poses.shape[0]
        zeta = torch.zeros(n, 6, dtype=torch.float64, requires_grad=True)
        pp = bt.perturb(po[fo:fo + n].detach().cpu().double(), zeta)
        L = _loss_torch(pp, do[fo:fo + n].detach().cpu().double(), p, cw)
        (gz,) = torch.autograd.grad(L, zeta)
        gpo[fo:fo + n, :6] = gz.float().cuda()
        gdo[fo:fo + n] = torch.from_numpy(cw[1]).float().cuda()
        fo += n
    torch.autograd.backward([po, do], [gpo, gdo])
    torch.cuda.synchronize()
    out = []
    fo = eo = 0
    for p in problems:
        n, e = p.poses.shape[0], p.ii.shape[0]
        out.append(dict(poses=poses.grad[fo:fo + n, :6].double().cpu().numpy(),
                        disps=disps.grad[fo:fo + n].double().cpu().numpy(),
                        targets=targets.grad[eo:eo + e].double().cpu().numpy(),
                        weights=weights.grad[eo:eo + e].double().cpu().numpy()))
        fo, eo = fo + n, eo + e
    return out


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _fd(p, cw, name, idx, h=1e-6):
    def loss_of(q):
        r = ob.ba(q, fp64=True)
        gt = p.poses_gt.double().numpy()
        err = W.se3_log(W.se3_mul(W.se3_inv(gt), r["poses"]))
        return float((cw[0] * err).sum() + (cw[1] * (r["disps"] - p.disps_gt.double().numpy())).sum())

    vals = []
    for s in (h, -h):
        q = p.clone()
        if name == "poses":
            n, k = idx
            P = p.poses.double().numpy().copy()
            xi = np.zeros(6)
            xi[k] = s
            P[n] = W.se3_mul(W.se3_exp(xi), P[n])
            q.poses = torch.from_numpy(P)
        else:
            t = getattr(p, name).double().clone()
            t[idx] += s
            setattr(q, name, t)
        vals.append(loss_of(q))
    return (vals[0] - vals[1]) / (2 * h)


def _picks(p, rng, n=8):
    N, H, W_ = p.disps.shape
    E = p.ii.shape[0]
    out = []
    for _ in range(n):
        out.append(("poses", (int(rng.integers(0, N)), int(rng.integers(0, 6)))))
        out.append(("disps", (int(rng.integers(0, N)), int(rng.integers(0, H)), int(rng.integers(0, W_)))))
        out.append(("targets", (int(rng.integers(0, E)), int(rng.integers(0, 2)), int(rng.integers(0, H)),
                                int(rng.integers(0, W_)))))
        out.append(("weights", (int(rng.integers(0, E)), int(rng.integers(0, 2)), int(rng.integers(0, H)),
                                int(rng.integers(0, W_)))))
    return out


def test_small_graph_adjoint_matches_torch_autograd_and_fd():
    p = _small_problem()
    cw = _loss_weights(p, 0)
    got = _cuda_grads([p], [cw])[0]
    want = _torch_grads(p, cw)
    for k in ("poses", "disps", "targets", "weights"):
        assert _rel(got[k], want[k]) < 2e-4, (k, _rel(got[k], want[k]))
    picks = _picks(p, np.random.default_rng(2))
    g = np.array([got[n][i] for n, i in picks])
    fd = np.array([_fd(p, cw, n, i) for n, i in picks])
    assert _rel(g, fd) < 1e-3, _rel(g, fd)


def test_training_window_adjoint_matches_torch_autograd_and_fd():
    probs = _window_problems()
    cws = [_loss_weights(p, 10 + c) for c, p in enumerate(probs)]
    got = _cuda_grads(probs, cws)
    rng = np.random.default_rng(3)
    for c, p in enumerate(probs):
        want = _torch_grads(p, cws[c])
        for k in ("poses", "disps", "targets", "weights"):
            assert _rel(got[c][k], want[k]) < 2e-4, (c, k, _rel(got[c][k], want[k]))
    p = probs[1]
    picks = _picks(p, rng)
    g = np.array([got[1][n][i] for n, i in picks])
    fd = np.array([_fd(p, cws[1], n, i) for n, i in picks])
    assert _rel(g, fd) < 1e-3, _rel(g, fd)


def test_forward_of_the_differentiable_solve_equals_the_plain_solve():
    probs = _window_problems()
    plan = BB.BatchPlan.for_problems(probs, "cuda", adjoint=True)
    batch = BB.concat_problems(probs, device="cuda")
    po, do = BA.bundle_adjust(plan, batch["poses"], batch["disps"], batch["targets"], batch["weights"],
                              batch["eta"], batch["disps_sens"], batch["intrinsics"], batch["ii"], batch["jj"],
                              batch["depth_active"], 2, 1e-4, 0.1)
    plain = {k: v.clone() for k, v in batch.items()}
    BB.BatchPlan.for_problems(probs, "cuda").solve(**plain, iterations=2, lm=1e-4, ep=0.1)
    assert torch.equal(po, plain["poses"]) and torch.equal(do, plain["disps"])
    assert not torch.equal(po, batch["poses"])  # inputs untouched, outputs moved
