"""The drop-in on backend-size graphs: large windows and depth frames coupled to many poses.

ViPE's backend runs bundle_adjustment(t0=1, t1=n_keyframes) over its whole keyframe
buffer (vipe/slam/components/factor_graph.py:376-392), with proximity and loop edges
that couple a keyframe's depth to many poses (:409-486).  The reference solves any
such window with a sparse Cholesky on the host (csrc/slam_ext/geom_kernels.cu:1269-1288).
Here:
  * depth frames coupled to more than 31 window poses take the wide-frame kernel
    (ba_frame_wide_kernel) instead of the tensor-core frame kernel;
  * reduced systems of more than 768 unknowns take the multi-launch blocked Cholesky.
Every case is held to the FP32 oracle (the reference's arithmetic) at the tolerances of
the other BA parity tests and, where stated, to the FP64 oracle at the north-star targets
(rotation 1e-4 rad, translation 1e-4 relative to the trajectory extent, depth 1e-3
relative median).  The graphs are built by vipe_b200.workloads.ba_backend.
"""

import numpy as np
import pytest
import torch

import oracle.ba as ob
from vipe_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _run_gpu(p, **kw):
    from vipe_b200.ext import slam_ext

    g = p.to("cuda")
    opt = dict(motion_only=False, optimize_intrinsics=False)
    opt.update(kw)
    dx, dz, en = slam_ext.ba_extended(g.poses, g.disps, g.intrinsics, g.disps_sens, g.targets, g.weights, g.eta, g.ii,
                                      g.jj, g.depth_active, g.t0, g.t1, g.iterations, g.lm, g.ep,
                                      opt["motion_only"], g.alpha, opt["optimize_intrinsics"], 1e-6, 1e-6, 1.0, True)
    torch.cuda.synchronize()
    assert not slam_ext.last_solver_failed()
    return dict(poses=g.poses.cpu().double().numpy(), disps=g.disps.cpu().double().numpy(),
                intrinsics=g.intrinsics.cpu().double().numpy(), dx=dx.cpu().double().numpy(),
                energy=en.cpu().double().numpy())


def _oracle(p, fp64, **kw):
    import os

    ob.set_threads(os.cpu_count() or 1)
    try:
        return ob.ba(p, fp64=fp64, compute_energy=True, **kw)
    finally:
        ob.set_threads(1)


def _close32(got, want32, want64):
    """FP32-oracle parity at the other BA tests' tolerances (poses 5e-5, depths 5e-4 abs + rel),
    widened to twice the FP32 oracle's own distance from the FP64 oracle where FP32 rounding of
    the larger systems exceeds them (the device sums pose blocks in FP64, the reference in FP32)."""
    pt = max(5e-5, 2 * np.abs(want32["poses"] - want64["poses"]).max())
    dt = max(5e-4, 2 * np.abs(want32["disps"] - want64["disps"]).max())
    np.testing.assert_allclose(got["poses"], want32["poses"], atol=pt, rtol=0)
    np.testing.assert_allclose(got["disps"], want32["disps"], atol=dt, rtol=5e-4)
    np.testing.assert_allclose(got["intrinsics"], want32["intrinsics"], atol=5e-5, rtol=1e-6)


def _quat_angle(q1, q2):
    d = np.abs(np.sum(q1 * q2, -1)) / (np.linalg.norm(q1, axis=-1) * np.linalg.norm(q2, axis=-1))
    return 2.0 * np.arccos(np.clip(d, -1.0, 1.0))


def _fp64_targets(got, want):
    gp, wp = got["poses"], want["poses"]
    assert _quat_angle(gp[:, 3:7], wp[:, 3:7]).max() <= 1e-4
    extent = np.linalg.norm(wp[:, :3] - wp[:1, :3], axis=-1).max()
    assert np.linalg.norm(gp[:, :3] - wp[:, :3], axis=-1).max() <= 1e-4 * extent
    rel = np.abs(got["disps"] - want["disps"]) / np.abs(want["disps"])
    assert np.median(rel) <= 1e-3


def test_backend_window_256_keyframes():
    """t0 = 1, t1 = 256 (a 1531-unknown reduced system: blocked Cholesky), 16 hub keyframes
    coupled to up to 52 window poses (wide frames), 24x32 depth (two pixel chunks per frame)."""
    p = W.ba_backend(256, ht=24, wd=32)
    slots = W.frame_slots(p)
    assert slots.max() > 40 and (slots > 31).sum() >= 8
    got = _run_gpu(p.clone())
    want32, want64 = _oracle(p, fp64=False), _oracle(p, fp64=True)
    _close32(got, want32, want64)
    _fp64_targets(got, want64)
    np.testing.assert_allclose(got["energy"], want32["energy"], rtol=1e-4)


def test_wide_frames_in_a_small_window():
    """64 keyframes (373 unknowns: the single-launch cluster Cholesky) with hubs coupled to 40+
    window poses: the wide-frame kernel beside the tensor-core frame kernel, full 48x64 depth."""
    p = W.ba_backend(64, hub_every=16, hub_degree=40, ht=48, wd=64, iterations=2, t0=2)
    assert (W.frame_slots(p) > 31).sum() >= 3
    got = _run_gpu(p.clone())
    want32, want64 = _oracle(p, fp64=False), _oracle(p, fp64=True)
    _close32(got, want32, want64)
    _fp64_targets(got, want64)


def test_long_window_without_wide_frames():
    """200 keyframes, band edges only (every frame within the tensor-core kernel's slots),
    a 1195-unknown reduced system: the blocked Cholesky alone."""
    p = W.make_ba_problem(200, W.band_edges(200, 3), seed=1006, ht=12, wd=16, t0=1, iterations=2,
                          intrinsics=(15.0, 15.0, 8.0, 6.0))
    assert W.frame_slots(p).max() <= 31
    got = _run_gpu(p.clone())
    want32, want64 = _oracle(p, fp64=False), _oracle(p, fp64=True)
    _close32(got, want32, want64)
    _fp64_targets(got, want64)


def test_backend_window_focal_and_motion_only():
    """The focal-length path (wide kernel with focal couplings, the focal row in the blocked
    Cholesky) and the motion-only path (no depth rows, blocked Cholesky) on a 160-keyframe window."""
    p = W.ba_backend(160, hub_every=20, hub_degree=36, ht=12, wd=16)
    got = _run_gpu(p.clone(), optimize_intrinsics=True)
    want = _oracle(p, fp64=False, optimize_intrinsics=True)
    np.testing.assert_allclose(got["poses"], want["poses"], atol=1e-4, rtol=0)
    np.testing.assert_allclose(got["disps"], want["disps"], atol=5e-4, rtol=5e-4)
    assert abs(got["intrinsics"][0] - p.intrinsics[0].item()) > 0
    np.testing.assert_allclose(got["intrinsics"], want["intrinsics"], atol=1e-4, rtol=0)
    got = _run_gpu(p.clone(), motion_only=True)
    want = _oracle(p, fp64=False, motion_only=True)
    np.testing.assert_allclose(got["poses"], want["poses"], atol=5e-5, rtol=0)
    np.testing.assert_array_equal(got["disps"], p.disps.double().numpy())

