"""Runs one named workload a few times on the current GPU (for profiling runs).

    python -m vipe_b200.run_case ba1 --reps 2        # 64 keyframes, 628 edges, 4 LM iterations
    python -m vipe_b200.run_case ba0                 # 8 keyframes, 26 edges, 2 LM iterations
    python -m vipe_b200.run_case corr_build --edges 64

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


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["ba0", "ba1", "corr_build"])
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--edges", type=int, default=64)
    a = ap.parse_args()
    if a.case in ("ba0", "ba1"):
        run_ba(a.case, a.reps)
    else:
        run_corr_build(a.edges, a.reps)
    print("ok")


if __name__ == "__main__":
    main()
