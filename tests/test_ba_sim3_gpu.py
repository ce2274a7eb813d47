"""Sim3 bundle adjustment on the GPU (batched plan with group "sim3").

Each clip of a Sim3 batch against the dense FP64 torch BA in its Sim3 form
(oracle/ba_torch.py): rotation 1e-4 rad, translation and scale 1e-4 relative,
depth 1e-3 relative (median), pose steps 1e-4 relative; the flow energy falls
over the iterations; plans refuse what the Sim3 form does not cover.
"""

import numpy as np
import pytest
import torch

from oracle import ba_torch as bt
from vipe_b200 import _lib
from vipe_b200 import ba_batch as BB
from vipe_b200 import workloads as W

pytestmark = pytest.mark.gpu

LM, EP, ITERS = 1e-4, 0.1, 3


def test_sim3_batch_matches_fp64_oracle():
    b = W.make_ba_batch(3, seed=17, frames_range=(8, 14), group="sim3", device="cuda")
    plan = BB.BatchPlan(*b.sizes, b.ht, b.wd, "cuda", group="sim3")
    t = {k: v.clone() for k, v in b.tensors.items()}
    dx, dz, en, st = plan.solve(**t, iterations=ITERS, lm=LM, ep=EP, compute_energy=True)
    torch.cuda.synchronize()
    assert st.cpu().tolist() == [0] * b.G
    en = en.cpu()
    assert bool((en[:, 1:] < en[:, :-1]).all()), en
    fo = po = 0
    for g in range(b.G):
        p = b.clip(g)
        out = bt.ba_torch(p.poses.double(), p.disps.double(), p.intrinsics.double(), p.disps_sens.double(),
                          p.targets.double(), p.weights.double(), p.eta.double(), p.ii, p.jj,
                          p.depth_active.double(), p.t0, p.t1, ITERS, LM, EP, p.alpha)
        n, P = b.num_frames[g], b.t1[g] - b.t0[g]
        got = t["poses"][fo:fo + n].double().cpu()
        want = out[0].detach()
        rot = float((got[:, 3:7] - want[:, 3:7]).abs().max()) * 2
        tr = float((got[:, :3] - want[:, :3]).abs().max() / want[:, :3].abs().max())
        sc = float(((got[:, 7] - want[:, 7]) / want[:, 7]).abs().max())
        gd = t["disps"][fo:fo + n].double().cpu()
        drel = float(((gd - out[1]).abs() / out[1].abs()).median())
        assert rot < 1e-4 and tr < 1e-4 and sc < 1e-4 and drel < 1e-3, (g, rot, tr, sc, drel)
        gx = dx[po:po + P].double().cpu()
        assert float((gx - out[2]).norm() / out[2].norm()) < 1e-3
        fo, po = fo + n, po + P


def test_sim3_plan_limits():
    b = W.make_ba_batch(2, seed=3, frames_range=(8, 10), group="sim3")
    plan = BB.BatchPlan(*b.sizes, b.ht, b.wd, "cuda", group="sim3")
    t = {k: v.cuda() for k, v in b.tensors.items()}
    with pytest.raises(RuntimeError):
        plan.solve(**t, iterations=1, lm=LM, ep=EP, optimize_intrinsics=True)
    with pytest.raises(RuntimeError, match="shape"):
        BB.BatchPlan(*b.sizes, b.ht, b.wd, "cuda").solve(**t, iterations=1, lm=LM, ep=EP)
