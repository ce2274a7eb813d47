"""Runs one named workload a few times on the current GPU (for profiling runs).

    python -m vipe_b200.run_case ba1 --reps 2        # 64 keyframes, 628 edges, 4 LM iterations
    python -m vipe_b200.run_case ba0                 # 8 keyframes, 26 edges, 2 LM iterations
    python -m vipe_b200.run_case corr_build --edges 64
    python -m vipe_b200.run_case batch --clips 32    # batched forward + adjoint, 4 LM iterations
    python -m vipe_b200.run_case lookup --edges 64   # radius-3 lookups: volume (4 levels) and indexed

Every repetition runs the full operation on fresh inputs; the process exits 0
only if every call returned success.
"""

from __future__ import annotations

import argparse

import torch


def run_ba(which: str, reps: int) -> None:
    from . import workloads as W
    from .ext import slam_ext

    p = W.ba_config1() if which == "ba1" else W.ba_config0()
    g0 = p.to("cuda")
    for _ in range(reps):
        q = g0.clone()
        slam_ext.ba_extended(q.poses, q.disps, q.intrinsics, q.disps_sens, q.targets, q.weights, q.eta, q.ii, q.jj,
                             q.depth_active, q.t0, q.t1, q.iterations, q.lm, q.ep, False, q.alpha, False, 1e-6, 1e-6,
                             1.0, False)
    torch.cuda.synchronize()


def run_corr_build(edges: int, reps: int) -> None:
    from .corr_build import corr_volume_pyramid

    C, H, Wd = 128, 48, 64
    g = torch.Generator(device="cuda").manual_seed(1002)
    f1 = (torch.randn(edges, C, H, Wd, generator=g, device="cuda") / C**0.5).to(torch.bfloat16)
    f2 = (torch.randn(edges, C, H, Wd, generator=g, device="cuda") / C**0.5).to(torch.bfloat16)
    for _ in range(reps):
        lv = corr_volume_pyramid(f1, f2, 4, out_dtype=torch.float16, check=True)
        del lv
    torch.cuda.synchronize()


def run_lookup(edges: int, reps: int) -> None:
    """FP16 pyramid of `edges` edges (128 ch, 48x64) looked up per level with corr_index_forward,
    then the indexed on-the-fly lookup of the same edges over 16 frames' FP16 maps."""
    import torch.nn.functional as F

    from .corr_build import corr_volume_pyramid
    from .ext import droid_net_ext as dne

    C, H, Wd, Nf = 128, 48, 64, 16
    g = torch.Generator(device="cuda").manual_seed(1002)
    f1 = (torch.randn(edges, C, H, Wd, generator=g, device="cuda") / C**0.5).to(torch.bfloat16)
    f2 = (torch.randn(edges, C, H, Wd, generator=g, device="cuda") / C**0.5).to(torch.bfloat16)
    lv = corr_volume_pyramid(f1, f2, 4, out_dtype=torch.float16, check=True)
    vols = [v.view(edges, H, Wd, H >> l, Wd >> l) for l, v in enumerate(lv)]
    yy, xx = torch.meshgrid(torch.arange(H, device="cuda"), torch.arange(Wd, device="cuda"), indexing="ij")
    coords = torch.stack([xx, yy], 0).float()[None] + 2.0 * torch.randn(edges, 2, 1, 1, generator=g, device="cuda")
    coords = (coords + torch.randn(edges, 2, H, Wd, generator=g, device="cuda")).contiguous()
    fm = (torch.randn(Nf, C, H, Wd, generator=g, device="cuda") / C**0.5).half() / 4.0
    pyr, t = [], fm
    for l in range(4):
        pyr.append(t.permute(0, 2, 3, 1).contiguous().view(1, Nf, H >> l, Wd >> l, C))
        t = F.avg_pool2d(t.float(), 2, stride=2).half()
    e = torch.arange(edges, device="cuda")
    ii, jj = e % Nf, (e % Nf + 1 + (e // Nf) % 7) % Nf
    c5 = coords.permute(0, 2, 3, 1).reshape(1, edges, H, Wd, 2).contiguous()
    for _ in range(reps):
        for l in range(4):
            dne.corr_index_forward(vols[l], (coords / 2**l).contiguous(), 3)
        dne.altcorr_index_forward(pyr[0], pyr, c5, ii, jj, 3)
    torch.cuda.synchronize()


def run_batch(clips: int, reps: int) -> None:
    from . import _lib
    from . import workloads as W
    from .ba_batch import BatchPlan

    b = W.make_ba_batch(clips, seed=1004, device="cuda")
    plan = BatchPlan(*b.sizes, b.ht, b.wd, "cuda", adjoint=True)
    it = 4
    tape = plan.make_tape(it)
    T = b.tensors
    g = torch.Generator(device="cuda").manual_seed(1005)
    for _ in range(reps):
        s = {k: v.clone() for k, v in T.items()}
        _, _, _, st = plan.solve(**s, iterations=it, lm=1e-4, ep=0.1, tape=tape)
        gp = torch.randn(plan.total_frames, 7, generator=g, device="cuda")
        gp[:, 6] = 0
        gd = torch.randn(plan.total_frames, b.ht, b.wd, generator=g, device="cuda")
        out = [torch.empty_like(T[k]) for k in ("targets", "weights", "eta", "disps_sens")]
        st2 = torch.zeros(plan.G, dtype=torch.int32, device="cuda")
        rc = _lib.load().vipe_slam_ba_batch_backward(
            plan._h, *[t.data_ptr() for t in tape], s["intrinsics"].data_ptr(), s["disps_sens"].data_ptr(),
            s["targets"].data_ptr(), s["weights"].data_ptr(), s["eta"].data_ptr(), s["ii"].data_ptr(),
            s["jj"].data_ptr(), s["depth_active"].data_ptr(), it, 1e-4, 0.1, 0.001, gp.data_ptr(), gd.data_ptr(),
            *[o.data_ptr() for o in out], st2.data_ptr(), torch.cuda.current_stream().cuda_stream)
        _lib.check(rc, "batch backward")
        torch.cuda.synchronize()
        if int(st.abs().sum()) or int(st2.abs().sum()):
            raise RuntimeError("device status set")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["ba0", "ba1", "corr_build", "batch", "lookup"])
    ap.add_argument("--clips", type=int, default=32)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--edges", type=int, default=64)
    a = ap.parse_args()
    if a.case in ("ba0", "ba1"):
        run_ba(a.case, a.reps)
    elif a.case == "batch":
        run_batch(a.clips, a.reps)
    elif a.case == "lookup":
        run_lookup(a.edges, a.reps)
    else:
        run_corr_build(a.edges, a.reps)
    print("ok")


if __name__ == "__main__":
    main()
