"""slam_ext — drop-in for the reference's ``vipe.ext.slam_ext`` pybind module.

Reference bindings: vipe csrc/slam_ext/slam.cpp:42-55.  Same names, positional
order, keyword names, defaults and return values; poses / disps / intrinsics are
mutated in place as in the reference.  All work runs in the vipe_b200 CUDA
library on the tensors' current stream.

Differences, all on inputs the reference does not define:
  * edge indices outside [0, num_frames) raise RuntimeError (the reference reads
    out of bounds);
  * a window with more than 127 poses (6*127+1 unknowns fill the shared-memory
    panel of the on-device Cholesky), or a depth frame coupled to more than 32
    window poses, raises RuntimeError (documented kernel limits);
  * frame_distance / projmap entries with out-of-range indices are NaN.
A Cholesky failure leaves dx = 0 silently, as in the reference
(geom_kernels.cu:1283-1285); ``last_solver_failed()`` reports it.
"""

from __future__ import annotations

import torch

from .. import _lib

# When True (default) each BA call reads the device status word once at the end
# (one stream synchronisation) and raises on device-detected errors.
CHECK_DEVICE_STATUS = True

_last_solver_failed = False


def last_solver_failed() -> bool:
    """True if the last checked BA call hit a non-positive-definite system."""
    return _last_solver_failed


def _check_ba_inputs(**tensors):
    for name, t in tensors.items():
        _lib.require_cuda(name, t)
        _lib.require_contiguous(name, t)


def ba_extended(
    poses,
    disps,
    intrinsics,
    disps_sens,
    targets,
    weights,
    eta,
    ii,
    jj,
    depth_active,
    t0,
    t1,
    iterations,
    lm,
    ep,
    motion_only,
    alpha,
    optimize_intrinsics,
    intrinsics_lm,
    intrinsics_ep,
    intrinsics_scale,
    compute_energy=False,
):
    """Bundle adjustment with ViPE's optional variables (reference slam.cpp:46-51).

    Returns [dx (t1-t0, 6), dz (|kx|, H*W) or None when motion_only,
    energy (iterations,) or (0,)].
    """
    _check_ba_inputs(
        targets=targets,
        weights=weights,
        poses=poses,
        disps=disps,
        intrinsics=intrinsics,
        disps_sens=disps_sens,
        ii=ii,
        jj=jj,
        depth_active=depth_active,
        eta=eta,
    )
    for name, t in (
        ("poses", poses),
        ("disps", disps),
        ("intrinsics", intrinsics),
        ("disps_sens", disps_sens),
        ("targets", targets),
        ("weights", weights),
        ("eta", eta),
        ("depth_active", depth_active),
    ):
        _lib.require_dtype(name, t, torch.float32)
    _lib.require_dtype("ii", ii, torch.int64)
    _lib.require_dtype("jj", jj, torch.int64)
    t0, t1, iterations = int(t0), int(t1), int(iterations)
    num_frames, ht, wd = disps.shape
    num_edges = ii.shape[0]
    num_kx = eta.shape[0]
    if tuple(poses.shape) != (num_frames, 7) or intrinsics.numel() < 4:
        raise RuntimeError("poses must be (N, 7) and intrinsics (4,)")
    if num_edges > 0 and (tuple(targets.shape) != (num_edges, 2, ht, wd) or tuple(weights.shape) != tuple(targets.shape)):
        raise RuntimeError("targets/weights must be (E, 2, H, W)")
    if jj.shape[0] != num_edges or depth_active.shape[0] < num_frames:
        raise RuntimeError("ii/jj/depth_active sizes do not match")
    dev = poses.device
    P = t1 - t0
    ws_bytes = _lib.load().vipe_slam_ba_workspace_size(num_frames, ht, wd, num_edges, num_kx, t0, t1)
    if ws_bytes == 0:
        if t0 < 0 or t1 <= t0 or t1 > num_frames:
            raise RuntimeError(f"invalid optimisation window t0={t0}, t1={t1} for {num_frames} frames")
        raise RuntimeError("bundle adjustment: unsupported sizes")
    with torch.cuda.device(dev):
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        dx = torch.zeros(max(P, 0), 6, dtype=torch.float32, device=dev)
        dz = None if motion_only else torch.empty(num_kx, ht * wd, dtype=torch.float32, device=dev)
        energy = torch.empty(iterations if compute_energy else 0, dtype=torch.float32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        rc = _lib.load().vipe_slam_ba_extended(
            poses.data_ptr(),
            disps.data_ptr(),
            intrinsics.data_ptr(),
            disps_sens.data_ptr(),
            _lib.ptr(targets),
            _lib.ptr(weights),
            eta.data_ptr(),
            _lib.ptr(ii),
            _lib.ptr(jj),
            depth_active.data_ptr(),
            num_frames,
            ht,
            wd,
            num_edges,
            num_kx,
            t0,
            t1,
            iterations,
            float(lm),
            float(ep),
            int(bool(motion_only)),
            float(alpha),
            int(bool(optimize_intrinsics)),
            float(intrinsics_lm),
            float(intrinsics_ep),
            float(intrinsics_scale),
            int(bool(compute_energy)),
            dx.data_ptr(),
            _lib.ptr(dz),
            energy.data_ptr() if compute_energy else None,
            ws.data_ptr(),
            ws_bytes,
            status.data_ptr(),
            _lib.stream_of(poses),
        )
        _lib.check(rc, "slam_ext.ba_extended")
        if CHECK_DEVICE_STATUS:
            _raise_device_status(int(status.item()), "slam_ext.ba_extended")
    return [dx, dz, energy]


def _raise_device_status(code: int, what: str) -> None:
    global _last_solver_failed
    _last_solver_failed = bool(code & _lib.VIPE_WARN_SOLVER)
    err = code & ~_lib.VIPE_WARN_SOLVER
    if err:
        raise RuntimeError(f"{what} failed on the device: {_lib.status_string(err)}")


def ba(
    poses,
    disps,
    intrinsics,
    disps_sens,
    targets,
    weights,
    eta,
    ii,
    jj,
    t0,
    t1,
    iterations,
    lm,
    ep,
    motion_only,
    alpha=0.05,
):
    """Legacy DROID bundle adjustment (reference slam.cpp:42-45, geom_kernels.cu:1826-1834):
    ba_extended with depth_active = 1, no focal optimisation and no energy."""
    _lib.require_cuda("disps", disps)
    depth_active = torch.ones(disps.shape[0], dtype=disps.dtype, device=disps.device)
    return ba_extended(
        poses,
        disps,
        intrinsics,
        disps_sens,
        targets,
        weights,
        eta,
        ii,
        jj,
        depth_active,
        t0,
        t1,
        iterations,
        lm,
        ep,
        motion_only,
        alpha,
        False,
        1e-6,
        1e-6,
        1.0,
        False,
    )


def frame_distance(poses, disps, intrinsics, pi, pj, qi, qj, di, beta):
    """Mean induced flow per frame pair (reference geom_kernels.cu:613-768, 1849-1877)."""
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics)):
        _lib.require_cuda(name, t)
        _lib.require_contiguous(name, t)
        _lib.require_dtype(name, t, torch.float32)
    for name, t in (("pi", pi), ("pj", pj), ("qi", qi), ("qj", qj), ("di", di)):
        _lib.require_cuda(name, t)
        _lib.require_contiguous(name, t)
        _lib.require_dtype(name, t, torch.int64)
    num = pi.shape[0]
    _, ht, wd = disps.shape
    dist = torch.zeros(num, dtype=torch.float32, device=poses.device)
    if num > 0:
        rc = _lib.load().vipe_slam_frame_distance(
            poses.data_ptr(), disps.data_ptr(), intrinsics.data_ptr(), pi.data_ptr(), pj.data_ptr(),
            qi.data_ptr(), qj.data_ptr(), di.data_ptr(), num, poses.shape[0], disps.shape[0],
            intrinsics.numel() // 4, ht, wd, float(beta), dist.data_ptr(),
            _lib.stream_of(poses),
        )
        _lib.check(rc, "slam_ext.frame_distance")
    return dist


def projmap(poses, disps, intrinsics, ii, jj):
    """Reprojection map (reference geom_kernels.cu:526-611, 1879-1903) -> [coords, valid]."""
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics)):
        _lib.require_cuda(name, t)
        _lib.require_contiguous(name, t)
        _lib.require_dtype(name, t, torch.float32)
    for name, t in (("ii", ii), ("jj", jj)):
        _lib.require_cuda(name, t)
        _lib.require_contiguous(name, t)
        _lib.require_dtype(name, t, torch.int64)
    num = ii.shape[0]
    _, ht, wd = disps.shape
    coords = torch.zeros(num, ht, wd, 3, dtype=torch.float32, device=poses.device)
    valid = torch.zeros(num, ht, wd, 1, dtype=torch.float32, device=poses.device)
    if num > 0:
        rc = _lib.load().vipe_slam_projmap(
            poses.data_ptr(), disps.data_ptr(), intrinsics.data_ptr(), ii.data_ptr(), jj.data_ptr(), num,
            min(poses.shape[0], disps.shape[0]), ht, wd, coords.data_ptr(), valid.data_ptr(), _lib.stream_of(poses),
        )
        _lib.check(rc, "slam_ext.projmap")
    return [coords, valid]


def depth_filter(poses, disps, intrinsics, ix, thresh):
    """Multi-view depth consistency count (reference geom_kernels.cu:770-885, 1905-1929)."""
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics), ("thresh", thresh)):
        _lib.require_cuda(name, t)
        _lib.require_contiguous(name, t)
        _lib.require_dtype(name, t, torch.float32)
    _lib.require_cuda("ix", ix)
    _lib.require_contiguous("ix", ix)
    _lib.require_dtype("ix", ix, torch.int64)
    num = ix.shape[0]
    nf, ht, wd = disps.shape
    nf = min(nf, poses.shape[0])
    counter = torch.zeros(num, ht, wd, dtype=torch.float32, device=disps.device)
    if num > 0:
        rc = _lib.load().vipe_slam_depth_filter(
            poses.data_ptr(), disps.data_ptr(), intrinsics.data_ptr(), ix.data_ptr(), thresh.data_ptr(), nf, num, ht,
            wd, counter.data_ptr(), _lib.stream_of(disps),
        )
        _lib.check(rc, "slam_ext.depth_filter")
    return counter


def iproj(poses, disps, intrinsics):
    """Back-projection to world points (reference geom_kernels.cu:887-953, 1931-1950)."""
    for name, t in (("poses", poses), ("disps", disps), ("intrinsics", intrinsics)):
        _lib.require_cuda(name, t)
        _lib.require_contiguous(name, t)
        _lib.require_dtype(name, t, torch.float32)
    nf, ht, wd = disps.shape
    if poses.shape[0] < nf:
        raise RuntimeError("iproj: poses has fewer rows than disps")
    points = torch.zeros(nf, ht, wd, 3, dtype=torch.float32, device=disps.device)
    rc = _lib.load().vipe_slam_iproj(
        poses.data_ptr(), disps.data_ptr(), intrinsics.data_ptr(), nf, ht, wd, points.data_ptr(),
        _lib.stream_of(disps),
    )
    _lib.check(rc, "slam_ext.iproj")
    return points
