"""The allocation-free bundle-adjustment entry point, through the C ABI.

vipe_slam_ba_extended_noalloc serves callers that cannot allocate device
memory (hosts that forbid allocation after start-up, and C/cgo/JNI bindings
with no CUDA allocator of their own).  It runs on a 32 MiB scratch array built
into the library instead of a caller-provided workspace.  These tests check
that it gives the same answer as vipe_slam_ba_extended on two calls in a row
(the second one reuses the scratch left by the first), that a call after one
that left NaN across the scratch is unaffected, and that a graph too large for
the scratch is refused before anything is launched.

The file name sorts last so that a stop-at-first-failure run has already run
every other test when it gets here.
"""

import numpy as np
import pytest
import torch

from vipe_b200 import _lib
from vipe_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _poisoned(p):
    """Problem `p` with NaN targets and weights: a solve of it leaves NaN across the scratch."""
    q = p.clone()
    q.targets.fill_(float("nan"))
    q.weights.fill_(float("nan"))
    return q


def _call(p, noalloc: bool, expect_ok: bool = True):
    """One ba_extended solve of problem `p` through the chosen C entry point."""
    lib = _lib.load()
    g = p.to("cuda")
    N, H, Wd = g.disps.shape
    E, K, P = g.ii.shape[0], g.eta.shape[0], g.t1 - g.t0
    dx = torch.zeros(P, 6, dtype=torch.float32, device="cuda")
    dz = torch.zeros(K, H * Wd, dtype=torch.float32, device="cuda")
    energy = torch.zeros(g.iterations, dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    args = [g.poses.data_ptr(), g.disps.data_ptr(), g.intrinsics.data_ptr(), g.disps_sens.data_ptr(),
            g.targets.data_ptr(), g.weights.data_ptr(), g.eta.data_ptr(), g.ii.data_ptr(), g.jj.data_ptr(),
            g.depth_active.data_ptr(), N, H, Wd, E, K, g.t0, g.t1, g.iterations, g.lm, g.ep, 0, g.alpha, 0, 1e-6,
            1e-6, 1.0, 1, dx.data_ptr(), dz.data_ptr(), energy.data_ptr()]
    stream = torch.cuda.current_stream().cuda_stream
    if noalloc:
        rc = lib.vipe_slam_ba_extended_noalloc(*args, status.data_ptr(), stream)
    else:
        ws_bytes = lib.vipe_slam_ba_workspace_size(N, H, Wd, E, K, g.t0, g.t1)
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
        rc = lib.vipe_slam_ba_extended(*args, ws.data_ptr(), ws_bytes, status.data_ptr(), stream)
    assert rc == 0, _lib.status_string(rc)
    torch.cuda.synchronize()
    if expect_ok:
        assert int(status.item()) == 0
    return {k: v.cpu().double().numpy() for k, v in
            dict(poses=g.poses, disps=g.disps, dx=dx, dz=dz, energy=energy).items()}


def _assert_same(got, want):
    # FP32 tolerances of the BA parity tests
    np.testing.assert_allclose(got["poses"], want["poses"], atol=5e-5, rtol=0)
    np.testing.assert_allclose(got["dx"], want["dx"], atol=5e-5, rtol=0)
    np.testing.assert_allclose(got["disps"], want["disps"], atol=5e-4, rtol=5e-4)
    np.testing.assert_allclose(got["dz"], want["dz"], atol=5e-4, rtol=5e-4)
    np.testing.assert_allclose(got["energy"], want["energy"], rtol=1e-4)


def test_noalloc_matches_workspace_entry_on_consecutive_calls():
    lib = _lib.load()
    assert lib.vipe_slam_ba_extended_noalloc is not None
    big, small = W.ba_config1(), W.ba_config0()  # 64 keyframes / 628 edges, then 8 / 26
    first = _call(big, noalloc=True)
    second = _call(small, noalloc=True)  # runs on the scratch the first call left behind
    _assert_same(first, _call(big, noalloc=False))
    _assert_same(second, _call(small, noalloc=False))


def test_noalloc_ignores_what_a_previous_call_left_in_the_scratch():
    """A solve of NaN inputs fills the shared scratch with NaN; a following good call must not read
    any of it (every scratch word it reads, it writes first)."""
    big, small = W.ba_config1(), W.ba_config0()
    _call(_poisoned(big), noalloc=True, expect_ok=False)
    after = _call(small, noalloc=True)
    for k, v in after.items():
        assert np.all(np.isfinite(v)), k
    _assert_same(after, _call(small, noalloc=False))


def test_noalloc_rejects_graph_beyond_scratch():
    lib = _lib.load()
    N, H, Wd, E = 64, 48, 64, 3000
    need = lib.vipe_slam_ba_workspace_size(N, H, Wd, E, N, 2, N)
    assert need > (32 << 20)
    poses = torch.zeros(N, 7, device="cuda")
    poses[:, 6] = 1
    disps = torch.ones(N, H, Wd, device="cuda")
    intr = torch.tensor([60.0, 60.0, 32.0, 24.0], device="cuda")
    tg = torch.zeros(E, 2, H, Wd, device="cuda")
    ii = torch.arange(E, device="cuda") % N
    jj = (ii + 1) % N
    eta = torch.ones(N, H, Wd, device="cuda")
    act = torch.ones(N, device="cuda")
    dx = torch.zeros(N - 2, 6, device="cuda")
    dz = torch.zeros(N, H * Wd, device="cuda")
    rc = lib.vipe_slam_ba_extended_noalloc(
        poses.data_ptr(), disps.data_ptr(), intr.data_ptr(), disps.data_ptr(), tg.data_ptr(), tg.data_ptr(),
        eta.data_ptr(), ii.data_ptr(), jj.data_ptr(), act.data_ptr(), N, H, Wd, E, N, 2, N, 1, 1e-4, 0.1, 0, 0.001,
        0, 1e-6, 1e-6, 1.0, 0, dx.data_ptr(), dz.data_ptr(), None, None, torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.VIPE_ERR_CAPACITY
    assert b"static scratch" in lib.vipe_last_error()
    torch.cuda.synchronize()
    assert torch.all(poses[:, :6] == 0)  # nothing ran
