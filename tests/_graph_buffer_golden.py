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


def robust_cases():
    return torch.load(GOLDEN, weights_only=False)["robust"]


def with_outliers(targets):
    """Config-0 targets (E, 2, H, W) with a deterministic ~2.7% of pixels moved by up to 15 px
    (small integers: the same bits on every machine)."""
    E, _, H, W = targets.shape
    idx = torch.arange(E * H * W).reshape(E, H, W)
    mask = (idx * 7919) % 37 == 0
    off = ((idx % 11).float() - 5.0) * 3.0
    t = targets.clone()
    t[:, 0] = torch.where(mask, t[:, 0] + off, t[:, 0])
    t[:, 1] = torch.where(mask, t[:, 1] - 0.5 * off + 4.0, t[:, 1])
    return t


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


def robust_setup(name):
    """(args, robust_kernel, threshold, mu_schedule) of a robust case: config 0's recorded
    ba_extended arguments with the outlier targets and the case's iteration count."""
    from vipe_b200.robust_ba import gnc_mu_schedule

    rc = robust_cases()[name]
    case = cases()["config0"]
    args = args_of(case)
    args[4] = with_outliers(args[4])
    args[12] = rc["iterations"]
    sched = None
    if rc["kernel"] == "gnc_tls":
        gnc = rc["gnc"]
        sched = gnc_mu_schedule(gnc["gnc_n_mu_steps"], gnc["gnc_gn_iters_per_mu"], gnc["gnc_mu_init"],
                                gnc["gnc_mu_step"], gnc["gnc_mu_max"])
        assert len(sched) == rc["iterations"]
    return case, args, rc["kernel"], rc["threshold"], sched


def assert_robust_matches_generic(name, poses, disps):
    """Poses within 2e-4, disparities within 3e-3 (mean 2e-4) of the generic solver.  The
    disparity bound is the non-robust config-0 one (2e-3, two iterations) widened for three
    iterations: the FP64 oracle sits 2.15e-3 from the generic solver on the Huber case too, so
    the gap is the generic solver's own FP32 rounding (measured max 2.15e-3 / 1.75e-3 /
    7.2e-4 for Huber / Tukey / GNC-TLS, means below 9e-5)."""
    rc = robust_cases()[name]
    n = rc["n_frames"]
    g = rc["generic"]
    torch.testing.assert_close(poses[:n].cpu().float(), g["poses"][:n], atol=2e-4, rtol=0)
    torch.testing.assert_close(disps[:n].cpu().float().clamp(min=0.001), g["disps"][:n], atol=3e-3, rtol=0)
    assert float((disps[:n].cpu().float().clamp(min=0.001) - g["disps"][:n]).abs().mean()) < 2e-4


def camera_cases():
    return torch.load(GOLDEN, weights_only=False)["camera"]


def camera_setup(name):
    """(case, args, kernel, threshold, k1) of an MEI-camera case: config 0's recorded arguments
    (outlier targets for the robust one) with the case's iteration count."""
    c = camera_cases()[name]
    case = cases()["config0"]
    args = args_of(case)
    if c["outliers"]:
        args[4] = with_outliers(args[4])
    args[12] = c["iterations"]
    return case, args, c["kernel"], c["threshold"], c["k1"]


def assert_camera_matches_generic(name, poses, disps):
    """Poses within 2e-4, disparities within 5e-3 (mean 2e-4) of the generic solver with the
    MEI camera; the FP64 oracle itself sits 2.5e-3 / 4.0e-3 (max) from it, the generic solver's
    FP32 rounding (means 1.4e-4 / 1.0e-4)."""
    c = camera_cases()[name]
    n = c["n_frames"]
    g = c["generic"]
    torch.testing.assert_close(poses[:n].cpu().float(), g["poses"][:n], atol=2e-4, rtol=0)
    d = disps[:n].cpu().float().clamp(min=0.001)
    torch.testing.assert_close(d, g["disps"][:n], atol=5e-3, rtol=0)
    assert float((d - g["disps"][:n]).abs().mean()) < 2e-4


# ---------------------------------------------------------------- multi-view rig case

RIG_T = (0.12, 0.02, -0.03)          # view 1's extrinsics (cam-to-central) translation
RIG_AA = (0.04, -0.09, 0.02)         # and axis-angle rotation; view 0 is the identity


def _quat_of_aa(aa):
    import math

    th = math.sqrt(sum(a * a for a in aa))
    s = math.sin(th / 2) / th
    return [aa[0] * s, aa[1] * s, aa[2] * s, math.cos(th / 2)]


def _mat(T):
    """(..., 7) [t, q] -> (..., 4, 4) float64."""
    T = T.double()
    x, y, z, w = T[..., 3], T[..., 4], T[..., 5], T[..., 6]
    R = torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                     2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                     2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1).reshape(*T.shape[:-1], 3, 3)
    M = torch.zeros(*T.shape[:-1], 4, 4, dtype=torch.float64)
    M[..., :3, :3] = R
    M[..., :3, 3] = T[..., :3]
    M[..., 3, 3] = 1
    return M


RIG_VIEW1_INTR = (1.07, 0.94, 0.9, -0.6)  # view 1 of the per-view case: fx, fy scale; cx, cy shift
RIG_ROT_ERR = (0.006, -0.004, 0.005)  # rig-rotation case: view 1's initial rotation error (axis-angle)


def rig_problem(outliers=False, views=False, rig_error=False):
    """A two-view rig built from config 0 (deterministic, CPU): keyframe poses, rig (2, 7), depth
    frames k * 2 + q (view 1: 0.9 x view 0), the expanded terms of config 0's edges (edge-major,
    view-minor, as GraphBuffer.expand_edge_multiview orders them), targets = the reprojection at
    the initial state through the rig plus a deterministic +-0.8 px pattern (optionally the
    outliers of with_outliers), config 0's weights per view, eta for kx, 2 LM iterations.
    views=True: per-view intrinsics (view 1: fx, fy scaled and cx, cy shifted by RIG_VIEW1_INTR;
    intrinsics (2, 4)) and two keyframe self-pairs (t0, t0) and (t0 + 1, t0 + 1), which expand
    to cross-view terms (k, q) -> (k, (q + 1) % 2) as GraphBuffer's default cross_view_idx does,
    so that source and target views (and intrinsics) differ within a term.
    rig_error=True: the returned rig (the solve's initial value) has view 1 rotated by
    RIG_ROT_ERR away from the rig the targets were made with (rig_true), for the solves that
    optimise the rig rotation."""
    import types

    from vipe_b200 import workloads as W

    p = W.ba_config0()
    N, H, Wd = p.disps.shape
    V = 2
    rig = torch.zeros(V, 7)
    rig[:, 6] = 1
    rig[1, :3] = torch.tensor(RIG_T)
    rig[1, 3:] = torch.tensor(_quat_of_aa(RIG_AA))
    disps = torch.stack([p.disps, 0.9 * p.disps], 1).reshape(N * V, H, Wd).contiguous()
    sens = torch.stack([p.disps_sens, p.disps_sens], 1).reshape(N * V, H, Wd).contiguous()
    kii, kjj, kw = p.ii, p.jj, p.weights
    intr = p.intrinsics.clone()
    if views:
        self_pairs = torch.tensor([p.t0, p.t0 + 1], dtype=p.ii.dtype)
        kii, kjj = torch.cat([p.ii, self_pairs]), torch.cat([p.jj, self_pairs])
        kw = torch.cat([p.weights, p.weights[:2]])
        sx, sy, ox, oy = RIG_VIEW1_INTR
        v1 = torch.tensor([intr[0] * sx, intr[1] * sy, intr[2] + ox, intr[3] + oy], dtype=intr.dtype)
        intr = torch.stack([intr, v1])
    E = kii.shape[0]
    pi = kii.repeat_interleave(V)
    pj = kjj.repeat_interleave(V)
    q = torch.arange(V).repeat(E)
    qj = torch.where(pi == pj, (q + 1) % V, q)
    di, dj = pi * V + q, pj * V + qj
    K = (intr if views else intr.reshape(1, 4).expand(V, 4)).double()
    G, Rg = _mat(p.poses), _mat(rig)
    T = torch.linalg.inv(Rg[qj]) @ G[pj] @ torch.linalg.inv(G[pi]) @ Rg[q]
    vv, uu = torch.meshgrid(torch.arange(H, dtype=torch.float64), torch.arange(Wd, dtype=torch.float64),
                            indexing="ij")
    uu, vv = uu.reshape(1, -1), vv.reshape(1, -1)
    Ki, Kj = K[q], K[qj]  # (E * V, 4): source view unprojects, target view projects
    X = torch.stack([(uu - Ki[:, 2:3]) / Ki[:, 0:1], (vv - Ki[:, 3:4]) / Ki[:, 1:2], torch.ones_like(uu).expand(
        E * V, -1)], 1)
    d = disps.double()[di].reshape(E * V, 1, -1)
    Pp = T[:, :3, :3] @ X + T[:, :3, 3:] * d
    z = Pp[:, 2].clamp(min=0.1)
    tu = Kj[:, 0:1] * Pp[:, 0] / z + Kj[:, 2:3]
    tv = Kj[:, 1:2] * Pp[:, 1] / z + Kj[:, 3:4]
    k = torch.arange(E * V, dtype=torch.float64)[:, None]
    pix = torch.arange(H * Wd, dtype=torch.float64)[None]
    tu = tu + 0.8 * torch.sin(0.37 * pix + 1.1 * k)
    tv = tv + 0.8 * torch.cos(0.23 * pix + 0.7 * k)
    targets = torch.stack([tu, tv], 1).reshape(E * V, 2, H, Wd).float()
    if outliers:
        targets = with_outliers(targets)
    weights = kw.repeat_interleave(V, 0).contiguous()
    kx = torch.unique(torch.cat([torch.arange(p.t0 * V, p.t1 * V), di]))
    disp_damping = ((p.eta.double() - 1e-7) / 0.2).float()  # per keyframe; both views share it
    eta_frames = disp_damping.repeat_interleave(V, 0)  # (N * V, H*W) in frame order
    eta = (0.2 * eta_frames[kx] + 1e-7).float().contiguous()
    rig_true = rig
    if rig_error:
        rig = rig.clone()
        e = _quat_of_aa(RIG_ROT_ERR)
        q1 = rig[1, 3:].double()
        # quaternion product e (x) q1: view 1's rotation with the error applied on the left
        x1, y1, z1, w1 = q1.tolist()
        x0, y0, z0, w0 = e
        rig[1, 3:] = torch.tensor([w0 * x1 + x0 * w1 + y0 * z1 - z0 * y1, w0 * y1 - x0 * z1 + y0 * w1 + z0 * x1,
                                   w0 * z1 + x0 * y1 - y0 * x1 + z0 * w1, w0 * w1 - x0 * x1 - y0 * y1 - z0 * z1],
                                  dtype=rig.dtype)
    return types.SimpleNamespace(poses=p.poses.clone(), rig=rig, rig_true=rig_true, disps=disps, disps_sens=sens,
                                 intrinsics=intr, targets=targets.contiguous(), weights=weights,
                                 ii=di.contiguous(), jj=dj.contiguous(), eta=eta, kx=kx,
                                 disp_damping=disp_damping, depth_active=torch.ones(N * V), t0=p.t0, t1=p.t1,
                                 iterations=2, lm=float(p.lm), ep=float(p.ep), alpha=float(p.alpha), N=N, V=V,
                                 pi=pi, pj=pj, q=q)


def rig_cases():
    return torch.load(GOLDEN, weights_only=False)["rig"]
