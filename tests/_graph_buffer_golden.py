"""Loads tests/golden/graph_buffer_fused_ba.pt (made by tests/golden/make_graph_buffer_fixtures.py).

Each case holds the arguments that the reference's `GraphBuffer._fused_ba`
(vipe/slam/components/buffer.py:364-489) passed to `slam_ext.ba_extended`, the
GraphBuffer state before the call, and the state that the reference's generic
torch solver reached on the same BA problem.  `replay` re-applies those
arguments through any `ba_extended` with the reference's positional order
(csrc/slam_ext/slam.cpp:42-51) and then the two steps that follow the call in
the reference: the intrinsics write-back (buffer.py:486-487) and
`disps.clamp_(min=0.001)` (buffer.py:563; the reference test's
`_run_fused_bundle_adjustment` does the same).
"""

from __future__ import annotations

import hashlib
from pathlib import Path

import torch

GOLDEN = Path(__file__).resolve().parent / "golden" / "graph_buffer_fused_ba.pt"
TOL = 2e-4  # the reference test's tolerance (tests/test_graph_buffer_fused_ba.py:191-194)


def cases():
    return torch.load(GOLDEN, weights_only=False)["cases"]


def _sha256(t):
    return hashlib.sha256(t.detach().cpu().contiguous().numpy().tobytes()).hexdigest()


def args_of(case):
    """The recorded ba_extended arguments (CPU tensors), with config 0's targets and weights
    regenerated by the workload generator and checked against the recorded digests."""
    args = list(case["args"])
    if case["kind"] == "config0":
        from vipe_b200 import workloads as W

        p = W.ba_config0()
        for k, i in (("targets", 4), ("weights", 5)):
            t = getattr(p, k)
            if _sha256(t) != case["digests"][k]:
                raise AssertionError(f"config-0 {k} differ from the ones the fixture was recorded with")
            args[i] = t
    return args


def replay(case, ba_extended, device):
    """Runs `ba_extended` on the recorded arguments the way GraphBuffer does; returns the final
    (poses, disps, intrinsics) buffers."""
    args = args_of(case)
    before = case["before"]
    poses = before["poses"].to(device).clone()
    disps = before["disps"].to(device).clone()
    intr_buf = before["intrinsics"].to(device).clone()
    assert torch.equal(args[0], before["poses"]) and torch.equal(args[1], before["disps"][:, 0])
    call = [poses, disps[:, 0]] + [a.to(device) if isinstance(a, torch.Tensor) else a for a in args[2:]]
    ba_extended(*call)
    if args[17]:  # optimize_intrinsics: GraphBuffer writes the solved 1/8-scale intrinsics back
        intr_buf[0, :4] = call[2] / args[20]
    disps.clamp_(min=0.001)
    return poses, disps, intr_buf


def assert_matches_generic(case, poses, disps, intr_buf, tol=TOL):
    n = case["n_frames"]
    g = case["generic"]
    torch.testing.assert_close(poses[:n].cpu().float(), g["poses"][:n], atol=tol, rtol=tol)
    torch.testing.assert_close(disps[:n].cpu().float(), g["disps"][:n], atol=tol, rtol=tol)
    torch.testing.assert_close(intr_buf.cpu().float(), g["intrinsics"], atol=tol, rtol=tol)
