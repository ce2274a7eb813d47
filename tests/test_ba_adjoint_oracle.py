"""The differentiable FP64 torch BA (oracle/ba_torch.py) against the C++ FP64 oracle.

Forward: same poses/disps/dx/dz as oracle/ba_oracle.cpp.  Backward: torch
autograd of the torch BA against FP64 central finite differences of the C++
oracle (h = 1e-6) on random entries of targets, weights, initial poses (left
tangent perturbations) and initial depths, for a random-weighted loss of pose
log-errors and depth errors.  With the damping differentiated the two agree to
about 1e-6 relative; with the damping held constant within 1e-3 (the size of
the term the CUDA adjoint therefore includes).
"""

import numpy as np
import pytest
import torch

import oracle.ba as ob
from oracle import ba_torch as bt
from vipe_b200 import workloads as W


def _problem():
    p = W.ba_small(n_frames=6, ht=12, wd=16, radius=2, seed=5, iterations=2, t0=2)
    # a stereo edge and an inactive depth frame, as the reference supports both
    p.ii = torch.cat([p.ii, torch.tensor([3])])
    p.jj = torch.cat([p.jj, torch.tensor([3])])
    p.targets = torch.cat([p.targets, p.targets[:1] + 0.3], 0)
    p.weights = torch.cat([p.weights, p.weights[:1]], 0)
    p.depth_active[4] = 0.0
    return p


def _loss_weights(p, seed=0):
    g = np.random.default_rng(seed)
    N, H, W_ = p.disps.shape
    return g.normal(size=(N, 6)), g.normal(size=(N, H, W_))


def _loss_np(poses, disps, p, cw):
    cp, cd = cw
    gt = p.poses_gt.double().numpy()
    err = W.se3_log(W.se3_mul(W.se3_inv(gt), poses))
    return float((cp * err).sum() + (cd * (disps - p.disps_gt.double().numpy())).sum())


def _loss_torch(poses, disps, p, cw):
    cp, cd = (torch.from_numpy(x) for x in cw)
    gt = p.poses_gt.double()
    err = bt.se3_log(bt.se3_mul(bt.se3_inv(gt), poses))
    return (cp * err).sum() + (cd * (disps - p.disps_gt.double())).sum()


def _oracle_loss(p, cw, **over):
    q = p.clone()
    for k, v in over.items():
        setattr(q, k, v)
    r = ob.ba(q, fp64=True)
    return _loss_np(r["poses"], r["disps"], p, cw)


def _autograd(p, cw, detach_damping):
    eps = torch.zeros(p.poses.shape[0], 6, dtype=torch.float64, requires_grad=True)
    d0 = p.disps.double().clone().requires_grad_(True)
    tg = p.targets.double().clone().requires_grad_(True)
    wt = p.weights.double().clone().requires_grad_(True)
    poses0 = bt.perturb(p.poses.double(), eps)
    out = bt.ba_torch(poses0, d0, p.intrinsics.double(), p.disps_sens.double(), tg, wt, p.eta.double(), p.ii, p.jj,
                      p.depth_active.double(), p.t0, p.t1, p.iterations, p.lm, p.ep, p.alpha,
                      detach_damping=detach_damping)
    L = _loss_torch(out[0], out[1], p, cw)
    L.backward()
    return dict(poses=eps.grad.numpy(), disps=d0.grad.numpy(), targets=tg.grad.numpy(), weights=wt.grad.numpy())


def _fd(p, cw, name, idx, h=1e-6):
    if name == "poses":
        n, k = idx
        base = p.poses.double().numpy()
        out = []
        for s in (h, -h):
            xi = np.zeros(6)
            xi[k] = s
            P = base.copy()
            P[n] = W.se3_mul(W.se3_exp(xi), base[n])
            out.append(_oracle_loss(p, cw, poses=torch.from_numpy(P)))
        return (out[0] - out[1]) / (2 * h)
    base = getattr(p, name).double()
    out = []
    for s in (h, -h):
        t = base.clone()
        t[idx] += s
        out.append(_oracle_loss(p, cw, **{name: t}))
    return (out[0] - out[1]) / (2 * h)


def test_torch_ba_matches_cpp_oracle_forward():
    p = _problem()
    want = ob.ba(p, fp64=True)
    out = bt.ba_torch(p.poses.double(), p.disps.double(), p.intrinsics.double(), p.disps_sens.double(),
                      p.targets.double(), p.weights.double(), p.eta.double(), p.ii, p.jj, p.depth_active.double(),
                      p.t0, p.t1, p.iterations, p.lm, p.ep, p.alpha)
    np.testing.assert_allclose(out[0].detach().numpy(), want["poses"], atol=1e-9)
    np.testing.assert_allclose(out[1].detach().numpy(), want["disps"], atol=1e-7)
    np.testing.assert_allclose(out[2].detach().numpy(), want["dx"], atol=1e-9)
    np.testing.assert_allclose(out[3].detach().numpy(), want["dz"], atol=1e-7)


@pytest.mark.parametrize("detach, tol", [(False, 1e-5), (True, 1e-3)])
def test_torch_autograd_matches_finite_differences(detach, tol):
    p = _problem()
    cw = _loss_weights(p)
    g = _autograd(p, cw, detach)
    rng = np.random.default_rng(1)
    picks = []
    N, H, W_ = p.disps.shape
    E = p.ii.shape[0]
    for _ in range(8):
        picks.append(("poses", (int(rng.integers(0, N)), int(rng.integers(0, 6)))))
        picks.append(("disps", (int(rng.integers(0, N)), int(rng.integers(0, H)), int(rng.integers(0, W_)))))
        picks.append(("targets", (int(rng.integers(0, E)), int(rng.integers(0, 2)), int(rng.integers(0, H)),
                                  int(rng.integers(0, W_)))))
        picks.append(("weights", (int(rng.integers(0, E)), int(rng.integers(0, 2)), int(rng.integers(0, H)),
                                  int(rng.integers(0, W_)))))
    ad = np.array([g[n][i] for n, i in picks])
    fd = np.array([_fd(p, cw, n, i) for n, i in picks])
    rel = np.linalg.norm(ad - fd) / np.linalg.norm(fd)
    assert rel < tol, (rel, list(zip([n for n, _ in picks], ad, fd)))
