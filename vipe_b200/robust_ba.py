"""Fused bundle adjustment with the generic solver's robust kernels.

The reference's fused path (GraphBuffer._fused_ba -> slam_ext.ba_extended) refuses robust
kernels (vipe/slam/components/buffer.py:531-547: "Fused BA is enabled, but robust kernels are
not supported") and falls back to the generic torch solver (vipe/slam/ba/solver.py,
terms.py, kernel.py) for them.  vipe_slam_ba_extended_robust runs them in the fused kernels:
every per-pixel linearisation multiplies the two flow channels' weights by the kernel of the
channel's residual at the linearisation point — exactly where the generic solver applies
``w <- w * kernel(r)`` (terms.py:73-75) — and the depth back-substitution keeps the rows of
pose t0 as the generic solver's Schur back-substitution does.

  ba_extended_robust(...)      the slam_ext.ba_extended arguments plus the kernel name,
                               threshold and, for GNC-TLS, the mu of every iteration, and the
                               camera model (pinhole, or MEI with its k1; the reference's fused
                               path takes pinhole only, buffer.py:387-388);
  ba_rig(...)                  the same over a multi-view rig: keyframe poses, fixed rig
                               extrinsics, depth frames k * n_views + q (the reference's fused
                               path takes single-view buffers with an identity rig only);
  gnc_mu_schedule(...)         the generic solver's GNC schedule (buffer.py:686-695: n_mu_steps
                               rounds of gn_iters_per_mu iterations, mu <- min(mu * step, max),
                               the hard TLS indicator once mu reaches its maximum).
"""

from __future__ import annotations

import math

import torch

from . import _lib
from .ext import slam_ext as _se

KINDS = {None: 0, "none": 0, "null": 0, "off": 0, "": 0, "huber": 1, "tukey": 2, "gnc_tls": 3, "gnc-tls": 3}


def gnc_mu_schedule(n_mu_steps=4, gn_iters_per_mu=6, mu_init=1.0, mu_step=1.4, mu_max=1.0e6):
    """Per-iteration mu of the generic solver's GNC loop; +inf marks the hard TLS indicator."""
    out, mu = [], float(mu_init)
    for _ in range(max(1, int(n_mu_steps))):
        for _ in range(max(1, int(gn_iters_per_mu))):
            out.append(math.inf if mu >= mu_max else mu)
        mu = min(mu * mu_step, mu_max)
    return out


CAMERAS = {None: 0, "pinhole": 0, "mei": 1}


def ba_extended_robust(poses, disps, intrinsics, disps_sens, targets, weights, eta, ii, jj, depth_active, t0, t1,
                       iterations, lm, ep, motion_only, alpha, optimize_intrinsics, intrinsics_lm, intrinsics_ep,
                       intrinsics_scale, compute_energy=False, robust_kernel=None, threshold=1.0,
                       mu_schedule=None, camera_type=None, distortion=0.0):
    """slam_ext.ba_extended with a robust kernel ('huber', 'tukey', 'gnc_tls' or None), the
    generic solver's back-substitution and the frames' camera model (camera_type 'pinhole' or
    'mei', with distortion = the MEI k1; a vipe CameraType's value works too).  Returns
    [dx, dz or None, energy]."""
    import ctypes

    cam_name = getattr(camera_type, "value", camera_type)
    cam_name = None if cam_name is None else str(cam_name).lower()
    if cam_name not in CAMERAS:
        raise ValueError(f"Unsupported camera_type for the fused BA: {camera_type!r}; expected 'pinhole' or 'mei'")
    cam = CAMERAS[cam_name]
    if cam == 1 and optimize_intrinsics:
        raise RuntimeError("optimize_intrinsics is not supported with the MEI camera")

    name = None if robust_kernel is None else str(robust_kernel).lower()
    if name not in KINDS:
        raise ValueError(f"Unknown robust_kernel: {robust_kernel!r}; expected 'huber' | 'tukey' | 'gnc_tls' | None")
    kind = KINDS[name]
    iterations = int(iterations)
    sched = None
    if kind == 3:
        if mu_schedule is None:
            raise RuntimeError("GNC-TLS needs the mu of every iteration (gnc_mu_schedule)")
        if len(mu_schedule) != iterations:
            raise RuntimeError("mu_schedule must hold one mu per iteration")
        sched = (ctypes.c_float * iterations)(*[float(m) for m in mu_schedule])
    elif kind != 0 and not float(threshold) > 0.0:
        raise RuntimeError("robust_threshold must be > 0")
    _se._check_ba_inputs(targets=targets, weights=weights, poses=poses, disps=disps, intrinsics=intrinsics,
                         disps_sens=disps_sens, ii=ii, jj=jj, depth_active=depth_active, eta=eta)
    for nm, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics), ("disps_sens", disps_sens),
                  ("targets", targets), ("weights", weights), ("eta", eta), ("depth_active", depth_active)):
        _lib.require_dtype(nm, t, torch.float32)
    _lib.require_dtype("ii", ii, torch.int64)
    _lib.require_dtype("jj", jj, torch.int64)
    t0, t1 = int(t0), int(t1)
    num_frames, ht, wd = disps.shape
    num_edges, num_kx = ii.shape[0], eta.shape[0]
    dev = poses.device
    lib = _lib.load()
    ws_bytes = lib.vipe_slam_ba_workspace_size(num_frames, ht, wd, num_edges, num_kx, t0, t1)
    if ws_bytes == 0:
        raise RuntimeError("robust bundle adjustment: unsupported sizes or window")
    with torch.cuda.device(dev):
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        dx = torch.zeros(max(t1 - t0, 0), 6, dtype=torch.float32, device=dev)
        dz = None if motion_only else torch.empty(num_kx, ht * wd, dtype=torch.float32, device=dev)
        energy = torch.empty(iterations if compute_energy else 0, dtype=torch.float32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        rc = lib.vipe_slam_ba_extended_generic(
            poses.data_ptr(), disps.data_ptr(), intrinsics.data_ptr(), disps_sens.data_ptr(), _lib.ptr(targets),
            _lib.ptr(weights), eta.data_ptr(), _lib.ptr(ii), _lib.ptr(jj), depth_active.data_ptr(), num_frames, ht,
            wd, num_edges, num_kx, t0, t1, iterations, float(lm), float(ep), int(bool(motion_only)), float(alpha),
            int(bool(optimize_intrinsics)), float(intrinsics_lm), float(intrinsics_ep), float(intrinsics_scale),
            int(bool(compute_energy)), dx.data_ptr(), _lib.ptr(dz), energy.data_ptr() if compute_energy else None,
            kind, float(threshold), None if sched is None else ctypes.cast(sched, ctypes.c_void_p), cam,
            float(distortion), ws.data_ptr(), ws_bytes, status.data_ptr(), _lib.stream_of(poses))
        _lib.check(rc, "ba_extended_robust")
        _se._raise_device_status(int(status.item()), "ba_extended_robust")
    return [dx, dz, energy]


def ba_rig(poses, rig, disps, intrinsics, disps_sens, targets, weights, eta, ii, jj, depth_active, t0, t1, iterations,
           lm, ep, motion_only, alpha, compute_energy=False, robust_kernel=None, threshold=1.0, mu_schedule=None,
           camera_type=None, distortion=0.0, optimize_rig_rotation=False, rig_damping=1e-4, rig_ep=1e-4):
    """Fused BA over a multi-view rig (vipe_slam_ba_rig): keyframe poses (N, 7), fixed rig
    extrinsics (V, 7), depth frames (N * V, H, W) indexed k * V + q, per-term source/target
    depth-frame indices ii, jj, and intrinsics (4,) shared by the views or (V, 4) per view (a
    term unprojects with its source view's row and projects with its target view's).
    distortion: the MEI k1 of every view, or a (V,) tensor with one per view.
    optimize_rig_rotation: the rotations of rig views 1..V-1 join the solve (the generic
    solver's rig group, buffer.py:668-673; rig_damping and rig_ep its damping) and are written
    back into ``rig``.  Returns [dx (t1 - t0, 6), dz or None, energy]."""
    import ctypes

    name = None if robust_kernel is None else str(robust_kernel).lower()
    if name not in KINDS:
        raise ValueError(f"Unknown robust_kernel: {robust_kernel!r}; expected 'huber' | 'tukey' | 'gnc_tls' | None")
    kind = KINDS[name]
    cam_name = getattr(camera_type, "value", camera_type)
    cam_name = None if cam_name is None else str(cam_name).lower()
    if cam_name not in CAMERAS:
        raise ValueError(f"Unsupported camera_type for the fused BA: {camera_type!r}; expected 'pinhole' or 'mei'")
    cam = CAMERAS[cam_name]
    iterations = int(iterations)
    sched = None
    if kind == 3:
        if mu_schedule is None or len(mu_schedule) != iterations:
            raise RuntimeError("GNC-TLS needs the mu of every iteration (gnc_mu_schedule)")
        sched = (ctypes.c_float * iterations)(*[float(m) for m in mu_schedule])
    _se._check_ba_inputs(targets=targets, weights=weights, poses=poses, rig=rig, disps=disps, intrinsics=intrinsics,
                         disps_sens=disps_sens, ii=ii, jj=jj, depth_active=depth_active, eta=eta)
    for nm, t in (("poses", poses), ("rig", rig), ("disps", disps), ("intrinsics", intrinsics),
                  ("disps_sens", disps_sens), ("targets", targets), ("weights", weights), ("eta", eta),
                  ("depth_active", depth_active)):
        _lib.require_dtype(nm, t, torch.float32)
    _lib.require_dtype("ii", ii, torch.int64)
    _lib.require_dtype("jj", jj, torch.int64)
    N, V = poses.shape[0], rig.shape[0]
    if disps.shape[0] != N * V:
        raise RuntimeError("disps must hold num_keyframes * n_views depth frames")
    if intrinsics.numel() == 4:
        intrinsics = intrinsics.reshape(1, 4).expand(V, 4).contiguous()
    elif tuple(intrinsics.shape) != (V, 4):
        raise RuntimeError("intrinsics must be (4,) or (n_views, 4)")
    t0, t1 = int(t0), int(t1)
    _, ht, wd = disps.shape
    num_edges, num_kx = ii.shape[0], eta.shape[0]
    dev = poses.device
    lib = _lib.load()
    opt = int(bool(optimize_rig_rotation))
    k1v = None
    if isinstance(distortion, torch.Tensor):
        k1v = distortion.to(device=poses.device, dtype=torch.float32).reshape(-1).contiguous()
        if k1v.numel() != V:
            raise RuntimeError("distortion must be a float or one value per view")
        if cam == 1 and not bool(((k1v >= 0) & (k1v <= 1)).all()):
            raise RuntimeError("MEI distortion must lie in [0, 1]")
        distortion = float(k1v[0])
    ws_bytes = lib.vipe_slam_ba_rig_workspace_size(N, V, ht, wd, num_edges, num_kx, t0, t1, opt)
    if ws_bytes == 0:
        raise RuntimeError("rig bundle adjustment: unsupported sizes or window")
    with torch.cuda.device(dev):
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        dx = torch.zeros(max(t1 - t0, 0), 6, dtype=torch.float32, device=dev)
        dz = None if motion_only else torch.empty(num_kx, ht * wd, dtype=torch.float32, device=dev)
        energy = torch.empty(iterations if compute_energy else 0, dtype=torch.float32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        rc = lib.vipe_slam_ba_rig(
            poses.data_ptr(), rig.data_ptr(), V, disps.data_ptr(), intrinsics.data_ptr(), disps_sens.data_ptr(),
            _lib.ptr(targets), _lib.ptr(weights), eta.data_ptr(), _lib.ptr(ii), _lib.ptr(jj), depth_active.data_ptr(),
            N, ht, wd, num_edges, num_kx, t0, t1, iterations, float(lm), float(ep), int(bool(motion_only)),
            float(alpha), int(bool(compute_energy)), dx.data_ptr(), _lib.ptr(dz),
            energy.data_ptr() if compute_energy else None, kind, float(threshold),
            None if sched is None else ctypes.cast(sched, ctypes.c_void_p), cam, float(distortion), _lib.ptr(k1v), opt,
            float(rig_damping), float(rig_ep), ws.data_ptr(), ws_bytes, status.data_ptr(), _lib.stream_of(poses))
        _lib.check(rc, "ba_rig")
        _se._raise_device_status(int(status.item()), "ba_rig")
    return [dx, dz, energy]
