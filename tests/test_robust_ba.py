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
