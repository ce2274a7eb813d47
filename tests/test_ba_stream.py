"""Streamed host batches (vipe_b200.ba_stream): the clip partition on CPU; on the
GPU, one streamed forward + backward step over pinned host tensors against one
plan over the whole batch with the same pixel chunking (per-graph arithmetic
does not depend on which graphs share a launch: bit-identical)."""

import random

import pytest
import torch

from vipe_b200.ba_stream import OUTPUT_KEYS, split_clips


@pytest.mark.parametrize("G", [1, 2, 3, 7, 64])
@pytest.mark.parametrize("parts", [1, 2, 4, 8, 100])
def test_split_clips_contiguous_and_nonempty(G, parts):
    rnd = random.Random(G * 1000 + parts)
    for _ in range(20):
        ne = [rnd.randint(0, 400) for _ in range(G)]
        for taper in (1.0, 0.25):
            r = split_clips(ne, parts, taper)
            assert len(r) == min(parts, G)
            assert r[0][0] == 0 and r[-1][1] == G
            assert all(a < b for a, b in r)
            assert all(r[i][1] == r[i + 1][0] for i in range(len(r) - 1))
        r = split_clips(ne, parts)
        assert len(r) == min(parts, G)
        assert r[0][0] == 0 and r[-1][1] == G
        assert all(a < b for a, b in r)
        assert all(r[i][1] == r[i + 1][0] for i in range(len(r) - 1))


def test_split_clips_balances_edges():
    ne = [100] * 64
    r = split_clips(ne, 8)
    assert [b - a for a, b in r] == [8] * 8


def test_split_clips_taper_shrinks_the_end_parts():
    ne = [100] * 64
    r = split_clips(ne, 8, taper=0.25)
    sizes = [b - a for a, b in r]
    assert len(sizes) == 8 and sum(sizes) == 64
    # the end parts hold about 0.25 / 6.5 of the edges each (cuts fall on whole graphs)
    assert max(sizes[0], sizes[-1]) <= 3
    assert all(s > max(sizes[0], sizes[-1]) for s in sizes[1:-1])
    assert split_clips(ne, 2, taper=0.25) == split_clips(ne, 2)  # fewer than 3 parts: no taper


@pytest.mark.gpu
def test_streamed_step_equals_one_plan():
    from vipe_b200 import workloads as W
    from vipe_b200.ba_batch import BATCH_KEYS, BatchPlan
    from vipe_b200.ba_stream import StreamedBundleAdjust

    b = W.make_ba_batch(10, seed=77, frames_range=(8, 24), device="cuda")
    it, lm, ep, alpha = 3, 1e-4, 0.1, 0.001
    ec, fc = 1, 2
    T = b.tensors
    g = torch.Generator(device="cuda").manual_seed(5)
    F = sum(b.num_frames)
    gin_p = torch.randn(F, 7, generator=g, device="cuda")
    gin_p[:, 6] = 0
    gin_d = torch.randn(F, b.ht, b.wd, generator=g, device="cuda")

    # one plan over the whole batch
    plan = BatchPlan(*b.sizes, b.ht, b.wd, "cuda", edge_chunks=ec, frame_chunks=fc, adjoint=True)
    s = {k: v.clone() for k, v in T.items()}
    tape = plan.make_tape(it)
    _, _, _, st = plan.solve(**s, iterations=it, lm=lm, ep=ep, alpha=alpha, tape=tape)
    gp, gd = gin_p.clone(), gin_d.clone()
    gt, gw = torch.empty_like(T["targets"]), torch.empty_like(T["weights"])
    ge, gs = torch.empty_like(T["eta"]), torch.empty_like(T["disps_sens"])
    st2 = torch.zeros(plan.G, dtype=torch.int32, device="cuda")
    plan.backward(tape, s["intrinsics"], s["disps_sens"], s["targets"], s["weights"], s["eta"], s["ii"], s["jj"],
                  s["depth_active"], it, lm, ep, alpha, gp, gd, gt, gw, ge, gs, st2)
    want = dict(poses=s["poses"], disps=s["disps"], grad_poses=gp, grad_disps=gd, grad_targets=gt, grad_weights=gw,
                grad_eta=ge, grad_disps_sens=gs)

    # streamed: three parts over pinned host tensors
    runner = StreamedBundleAdjust(b.sizes, b.ht, b.wd, "cuda", parts=3, iterations=it, lm=lm, ep=ep, alpha=alpha,
                                  edge_chunks=ec, frame_chunks=fc)
    assert len(runner.parts) == 3
    host = {k: T[k].cpu().pin_memory() for k in BATCH_KEYS}
    hp, hd = gin_p.cpu().pin_memory(), gin_d.cpu().pin_memory()
    out = runner.host_outputs()
    runner.step(host, hp, hd, out)
    torch.cuda.current_stream().synchronize()
    assert int(st.abs().sum()) == 0 and int(st2.abs().sum()) == 0
    assert int(runner.status().abs().sum()) == 0
    for k in OUTPUT_KEYS:
        torch.testing.assert_close(out[k], want[k].cpu(), rtol=0, atol=0, msg=k)


@pytest.mark.gpu
def test_streamed_forward_only_equals_one_plan():
    from vipe_b200 import workloads as W
    from vipe_b200.ba_batch import BATCH_KEYS, BatchPlan
    from vipe_b200.ba_stream import StreamedBundleAdjust

    b = W.make_ba_batch(9, seed=78, frames_range=(8, 24), device="cuda")
    it, lm, ep = 3, 1e-4, 0.1
    T = b.tensors
    plan = BatchPlan(*b.sizes, b.ht, b.wd, "cuda", edge_chunks=2, frame_chunks=1)
    s = {k: v.clone() for k, v in T.items()}
    plan.solve(**s, iterations=it, lm=lm, ep=ep)
    runner = StreamedBundleAdjust(b.sizes, b.ht, b.wd, "cuda", parts=4, iterations=it, lm=lm, ep=ep, edge_chunks=2,
                                  frame_chunks=1, adjoint=False)
    host = {k: T[k].cpu().pin_memory() for k in BATCH_KEYS}
    out = runner.host_outputs()
    assert set(out) == {"poses", "disps"}
    runner.step(host, None, None, out)
    torch.cuda.current_stream().synchronize()
    torch.testing.assert_close(out["poses"], s["poses"].cpu(), rtol=0, atol=0)
    torch.testing.assert_close(out["disps"], s["disps"].cpu(), rtol=0, atol=0)
