"""Host-side checks of vipe_b200.robust_ba (no GPU): kernel names, the GNC schedule and the
argument errors that precede any device work."""

import math

import pytest
import torch

from vipe_b200 import robust_ba as R


def test_gnc_schedule_follows_the_generic_solver_loop():
    # buffer.py:686-695: n_mu_steps rounds of gn_iters_per_mu iterations, mu <- min(mu * step, max),
    # hard indicator (mu >= mu_max) -> +inf
    assert R.gnc_mu_schedule(2, 2, 1.0, 3.0, 3.0) == [1.0, 1.0, math.inf, math.inf]
    s = R.gnc_mu_schedule(4, 6, 1.0, 1.4, 1.0e6)
    assert len(s) == 24 and s[0] == 1.0 and abs(s[6] - 1.4) < 1e-12 and abs(s[23] - 1.4**3) < 1e-9
    assert R.gnc_mu_schedule(0, 0) == [1.0]  # max(1, .) like the reference


def _dummy():
    z = torch.zeros(1)
    return [z] * 10 + [0, 1, 2, 1e-4, 0.1, False, 1e-3, False, 0.0, 0.0, 1.0]


def test_unknown_kernel_name_raises_value_error():
    with pytest.raises(ValueError, match="Unknown robust_kernel"):
        R.ba_extended_robust(*_dummy(), robust_kernel="cauchy")


def test_gnc_needs_one_mu_per_iteration():
    with pytest.raises(RuntimeError, match="mu of every iteration"):
        R.ba_extended_robust(*_dummy(), robust_kernel="gnc_tls")
    with pytest.raises(RuntimeError, match="one mu per iteration"):
        R.ba_extended_robust(*_dummy(), robust_kernel="gnc_tls", mu_schedule=[1.0])


def test_threshold_must_be_positive():
    with pytest.raises(RuntimeError, match="> 0"):
        R.ba_extended_robust(*_dummy(), robust_kernel="huber", threshold=0.0)


def test_cpu_tensors_are_refused():
    with pytest.raises(RuntimeError):
        R.ba_extended_robust(*_dummy(), robust_kernel="huber", threshold=1.0)


def test_unknown_camera_raises():
    with pytest.raises(ValueError, match="camera_type"):
        R.ba_extended_robust(*_dummy(), camera_type="panorama")


def test_rig_workspace_covers_the_rig_rotation_solve():
    """Host-only sizing of the rig solve: optimising the rig rotation makes every (keyframe, view)
    a virtual unknown and adds six rows per optimised view, so its workspace is larger; a rig
    whose keyframes x views exceed the solver's 1024 window poses is refused (size 0)."""
    from vipe_b200 import _lib

    lib = _lib.load()
    N, V, H, W, E, K, t0, t1 = 40, 3, 48, 64, 300, 120, 30, 40
    fixed = lib.vipe_slam_ba_rig_workspace_size(N, V, H, W, E, K, t0, t1, 0)
    rot = lib.vipe_slam_ba_rig_workspace_size(N, V, H, W, E, K, t0, t1, 1)
    assert fixed > 0 and rot > fixed
    # 400 keyframes x 3 views = 1200 virtual unknowns: fine with a fixed rig (window 30 x 3), not
    # when the rig rotation is optimised
    assert lib.vipe_slam_ba_rig_workspace_size(400, V, H, W, E, K, t0, t1, 0) > 0
    assert lib.vipe_slam_ba_rig_workspace_size(400, V, H, W, E, K, t0, t1, 1) == 0
    # one view: the rig has nothing to optimise (view 0 is fixed), so the flag changes nothing
    assert lib.vipe_slam_ba_rig_workspace_size(N, 1, H, W, E, 40, t0, t1, 1) == \
        lib.vipe_slam_ba_rig_workspace_size(N, 1, H, W, E, 40, t0, t1, 0)
