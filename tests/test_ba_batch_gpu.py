"""Batched BA on the GPU: many uneven clips in one solve (vipe_b200.ba_batch).

Each clip of a batch must give what the single-graph drop-in gives on that clip
alone (same kernels, FP32 tolerance of the drop-in tests: poses atol 5e-5,
disps atol/rtol 5e-4, focal rtol 2e-5); a CUDA-graph replay must reproduce the eager batched
solve bit for bit; a bad graph must be reported in its own status word without
touching the others; and the batch must stay within the FP64-oracle accuracy
bar (rotation 1e-4 rad, translation 1e-4 relative, depth 1e-3 relative median).
"""

import numpy as np
import pytest
import torch

import oracle.ba as ob
from vipe_b200 import _lib
from vipe_b200 import ba_batch as BB
from vipe_b200 import workloads as W

pytestmark = pytest.mark.gpu

LM, EP, ITERS = 1e-4, 0.1, 2


def _batch(num=5, seed=11, frames=(8, 20)):
    return W.make_ba_batch(num, seed=seed, frames_range=frames, device="cuda")


def _solve_batched(b, **kw):
    plan = BB.BatchPlan(*b.sizes, b.ht, b.wd, "cuda", **{k: kw.pop(k) for k in ("edge_chunks", "frame_chunks")
                                                          if k in kw})
    t = {k: v.clone() for k, v in b.tensors.items()}
    dx, dz, en, st = plan.solve(**t, iterations=ITERS, lm=LM, ep=EP, **kw)
    torch.cuda.synchronize()
    return t, dx, dz, en, st


def _solve_single(p, **kw):
    from vipe_b200.ext import slam_ext

    g = p.to("cuda")
    dx, dz, en = slam_ext.ba_extended(g.poses, g.disps, g.intrinsics, g.disps_sens, g.targets, g.weights, g.eta,
                                      g.ii, g.jj, g.depth_active, g.t0, g.t1, ITERS, LM, EP,
                                      kw.get("motion_only", False), g.alpha, kw.get("optimize_intrinsics", False),
                                      1e-6, 1e-6, kw.get("intrinsics_scale", 1.0), kw.get("compute_energy", False))
    torch.cuda.synchronize()
    return g, dx, dz, en


@pytest.mark.parametrize("opts", [dict(), dict(motion_only=True), dict(optimize_intrinsics=True,
                                                                       intrinsics_scale=0.125, compute_energy=True)])
def test_batch_matches_single_graph_calls(opts):
    b = _batch()
    t, dx, dz, en, st = _solve_batched(b, **opts)
    assert st.cpu().tolist() == [0] * b.G
    fo = eo = ko = po = 0
    for g in range(b.G):
        p = b.clip(g)
        s, sdx, sdz, sen = _solve_single(p, **opts)
        n, k, P = b.num_frames[g], b.num_kx[g], b.t1[g] - b.t0[g]
        torch.testing.assert_close(t["poses"][fo:fo + n], s.poses, atol=5e-5, rtol=0)
        torch.testing.assert_close(t["disps"][fo:fo + n], s.disps, atol=5e-4, rtol=5e-4)
        # the focal update sums every edge pixel; other chunkings change its FP32 order
        torch.testing.assert_close(t["intrinsics"][g], s.intrinsics, atol=5e-5, rtol=2e-5)
        torch.testing.assert_close(dx[po:po + P], sdx, atol=5e-5, rtol=0)
        if not opts.get("motion_only"):
            torch.testing.assert_close(dz[ko:ko + k], sdz, atol=5e-4, rtol=5e-4)
        if opts.get("compute_energy"):
            torch.testing.assert_close(en[g], sen, rtol=1e-4, atol=0)
        fo, ko, po = fo + n, ko + k, po + P


def test_batch_of_one_is_bitwise_the_single_call():
    b = _batch(num=1, seed=5, frames=(30, 30))
    p = b.clip(0)
    s, sdx, sdz, _ = _solve_single(p)
    # the single call picks its chunking for a graph alone; force the same
    from vipe_b200 import _lib as L  # noqa: F401
    E, K = b.num_edges[0], b.num_kx[0]
    che = max(1, min((296 + E - 1) // E, max(1, 48 * 64 // 1024)))
    cf = max(1, min((296 + K - 1) // K, 8))
    t, dx, dz, _, st = _solve_batched(b, edge_chunks=che, frame_chunks=cf)
    assert int(st[0]) == 0
    assert torch.equal(t["poses"], s.poses) and torch.equal(t["disps"], s.disps)
    assert torch.equal(dx, sdx) and torch.equal(dz, sdz)


def test_cuda_graph_replay_is_bitwise_eager():
    b = _batch(num=4, seed=21)
    plan = BB.BatchPlan(*b.sizes, b.ht, b.wd, "cuda")
    eager = {k: v.clone() for k, v in b.tensors.items()}
    dx0, dz0, _, _ = plan.solve(**eager, iterations=ITERS, lm=LM, ep=EP)
    static = {k: v.clone() for k, v in b.tensors.items()}
    cap = plan.capture(static, iterations=ITERS, lm=LM, ep=EP)
    for _ in range(2):  # replays restart from fresh inputs copied into the static tensors
        for k in ("poses", "disps", "intrinsics"):
            static[k].copy_(b.tensors[k])
        dx1, dz1, _, st = cap.replay()
        torch.cuda.synchronize()
        assert torch.equal(static["poses"], eager["poses"]) and torch.equal(static["disps"], eager["disps"])
        assert torch.equal(dx1, dx0) and torch.equal(dz1, dz0)
        assert st.cpu().tolist() == [0] * b.G


def test_bad_graph_is_reported_in_its_own_status():
    b = _batch(num=3, seed=4)
    t = {k: v.clone() for k, v in b.tensors.items()}
    e1 = b.num_edges[0]
    t["ii"][e1 + 2] = b.num_frames[1] + 5  # graph 1: an index past its frames
    plan = BB.BatchPlan(*b.sizes, b.ht, b.wd, "cuda")
    poses_before = t["poses"].clone()
    _, _, _, st = plan.solve(**t, iterations=ITERS, lm=LM, ep=EP)
    st = st.cpu().tolist()
    assert st[0] == 0 and st[2] == 0 and st[1] == _lib.VIPE_ERR_INDEX
    f0, f1 = b.num_frames[0], b.num_frames[1]
    assert torch.equal(t["poses"][f0:f0 + f1], poses_before[f0:f0 + f1])  # untouched
    assert not torch.equal(t["poses"][:f0], poses_before[:f0])


def test_batch_accuracy_against_fp64_oracle():
    b = _batch(num=3, seed=31, frames=(10, 16))
    t, *_ = _solve_batched(b)
    fo = 0
    for g in range(b.G):
        p = b.clip(g)
        p.iterations = ITERS
        want = ob.ba(p, fp64=True)
        n = b.num_frames[g]
        got_p = t["poses"][fo:fo + n].double().cpu().numpy()
        got_d = t["disps"][fo:fo + n].double().cpu().numpy()
        rot = np.abs(got_p[:, 3:] - want["poses"][:, 3:]).max() * 2  # quaternion -> angle (small)
        ext = np.abs(want["poses"][:, :3]).max()
        tr = np.abs(got_p[:, :3] - want["poses"][:, :3]).max() / ext
        drel = np.median(np.abs(got_d - want["disps"]) / np.abs(want["disps"]))
        assert rot < 1e-4 and tr < 1e-4 and drel < 1e-3, (g, rot, tr, drel)
        fo += n


def test_autotune_picks_a_measured_candidate():
    b = _batch(num=6, seed=8)
    res = BB.autotune(b.sizes, b.ht, b.wd, b.tensors, ITERS, LM, EP, "cuda", candidates=((1, 1), (2, 2)), reps=1)
    assert (res.edge_chunks, res.frame_chunks) in ((1, 1), (2, 2))
    assert len(res.table) == 2 and res.ms == min(x[2] for x in res.table)
    t, *_ = _solve_batched(b, edge_chunks=res.edge_chunks, frame_chunks=res.frame_chunks)
    t2, *_ = _solve_batched(b)
    torch.testing.assert_close(t["poses"], t2["poses"], atol=5e-5, rtol=0)
