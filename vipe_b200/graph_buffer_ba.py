"""GraphBuffer.bundle_adjustment on the fused GPU solver for the generic path's configurations.

The reference's GraphBuffer.bundle_adjustment (vipe/slam/components/buffer.py:501-700) takes
the fused CUDA solver only for single-view pinhole buffers with an identity rig and no robust
kernel (buffer.py:387-404, 541-545); everything else goes to the generic torch solver
(vipe/slam/ba/solver.py, terms.py).  `bundle_adjustment` here is a drop-in for that method
that runs those configurations on this library's fused kernels:

  * multi-view rigs (n_views > 1, per-view intrinsics and MEI distortion, rig extrinsics fixed
    or with their rotations optimised as the generic solver's rig group): vipe_slam_ba_rig;
  * robust kernels (Huber, Tukey, GNC-TLS with its mu schedule) and the MEI camera:
    vipe_slam_ba_extended_generic / vipe_slam_ba_rig;
  * single-view pinhole buffers with focal optimisation as before.

(With one view optimize_rig_rotation changes nothing: the generic solver fixes rig 0.) It raises
for what it does not cover: focal/distortion optimisation with MEI or with a rig, panorama
cameras, and sparse tracks together with a robust kernel.  Install with

    GraphBuffer.bundle_adjustment = vipe_b200.graph_buffer_ba.bundle_adjustment
"""

from __future__ import annotations

import torch

from . import robust_ba as R

WEIGHT_SCALE = 0.001  # the dense-flow and sparse-track weights of the generic path (buffer.py:524)


def robust_settings(ba_config, n_iters):
    """(kind name, threshold, mu schedule or None, iterations) of the buffer's BA config, with the
    generic solver's GNC loop (buffer.py:686-695) unrolled into one mu per iteration."""
    name = ba_config.get("robust_kernel", None)
    name = None if name is None else str(name).lower()
    if name in ("none", "null", "off", ""):
        name = None
    thr = float(ba_config.get("robust_kernel_threshold", 1.0))
    if name in ("gnc_tls", "gnc-tls"):
        sched = R.gnc_mu_schedule(int(ba_config.get("gnc_n_mu_steps", 4)), int(ba_config.get("gnc_gn_iters_per_mu", 6)),
                                  float(ba_config.get("gnc_mu_init", 1.0)), float(ba_config.get("gnc_mu_step", 1.4)),
                                  float(ba_config.get("gnc_mu_max", 1.0e6)))
        return name, thr, sched, len(sched)
    return name, thr, None, int(n_iters)


def bundle_adjustment(self, target, weight, disp_damping, ii, jj, t0, t1, n_iters, pose_damping, pose_ep,
                      motion_only, limited_disp, optimize_intrinsics, optimize_rig_rotation, verbose=False):
    """Drop-in for GraphBuffer.bundle_adjustment (same arguments) on the fused GPU solver."""
    cam = getattr(self.camera_type, "value", self.camera_type)
    cam = str(cam).lower()
    if cam not in ("pinhole", "mei"):
        raise RuntimeError(f"fused BA: camera type {cam!r} is not supported")
    V = int(self.n_views)
    kernel, thr, sched, iters = robust_settings(self.ba_config, n_iters)
    pi, qi, di, pj, qj, dj = self.expand_edge_multiview(ii, jj)
    H, W = self.height // 8, self.width // 8
    n_terms = di.shape[0]
    target = target.reshape(n_terms, H * W, 2)
    weight = weight.reshape(n_terms, H * W, 2)
    if self.sparse_tracks.enabled:
        if kernel is not None:
            raise RuntimeError("fused BA: sparse tracks with a robust kernel are not supported")
        st, sw = self.sparse_tracks.compute_dense_disp_target_weight(
            source_view_inds=qi, source_frame_inds=self.tstamp[pi], target_view_inds=qj,
            target_frame_inds=self.tstamp[pj], image_size=(self.height, self.width), dense_disp_size=(H, W))
        st, sw = st.flatten(1, 2), sw.flatten(1, 2)
        cw = weight + sw
        target = torch.where(cw > 0, (weight * target + sw * st) / cw.clamp_min(1e-12), target)
        weight = cw
    target = target.reshape(n_terms, H, W, 2).permute(0, 3, 1, 2).contiguous()
    weight = weight.reshape(n_terms, H, W, 2).permute(0, 3, 1, 2).contiguous()
    intr = self.intrinsics
    k1 = float(intr[0, 4]) if cam == "mei" else 0.0
    intr8 = (intr[0, :4] / 8.0).contiguous()
    nv = self.disps.shape[0] * V
    disps = self.disps.view(nv, H, W)
    sens = self.disps_sens.reshape(nv, H, W).contiguous()
    dd = disp_damping.reshape(nv, H * W)
    depth_active = torch.ones(nv, dtype=disps.dtype, device=disps.device)
    if limited_disp:
        depth_active.zero_()
        depth_active[t0 * V:t1 * V] = 1.0
    kx = torch.unique(torch.cat([torch.arange(t0 * V, t1 * V, device=di.device), di]))
    eta = (0.2 * dd[kx] + 1e-7).contiguous()
    identity = torch.tensor([0, 0, 0, 0, 0, 0, 1], dtype=self.rig.dtype, device=self.rig.device)
    single = V == 1 and torch.allclose(self.rig[0], identity)
    alpha = float(self.ba_config.dense_disp_alpha)
    if single:
        if torch.any(di == dj):
            raise RuntimeError("fused BA: self edges are not supported")
        R.ba_extended_robust(self.poses, disps, intr8, sens, target, weight, eta, di.contiguous(), dj.contiguous(),
                             depth_active, t0, t1, iters, pose_damping, pose_ep, motion_only, alpha,
                             optimize_intrinsics, 1e-6 * self.ba_config.get("intrinsics_damping_scale", 1.0),
                             1e-6 * self.ba_config.get("intrinsics_damping_scale", 1.0), 1.0 / 8.0, verbose,
                             robust_kernel=kernel, threshold=thr, mu_schedule=sched, camera_type=cam,
                             distortion=k1)
        if optimize_intrinsics:
            self.intrinsics[0, :4] = intr8 * 8.0
    else:
        if optimize_intrinsics:
            raise RuntimeError("fused BA: intrinsics optimisation with a rig is not supported")
        if torch.any(di == dj):
            raise RuntimeError("fused BA: terms within one depth frame are not supported")
        intr8v = (intr[:, :4] / 8.0).float().contiguous()  # one row per view
        rig = self.rig.float().contiguous()
        R.ba_rig(self.poses, rig, disps, intr8v, sens, target, weight, eta, di.contiguous(),
                 dj.contiguous(), depth_active, t0, t1, iters, pose_damping, pose_ep, motion_only, alpha, verbose,
                 robust_kernel=kernel, threshold=thr, mu_schedule=sched, camera_type=cam,
                 distortion=intr[:, 4].float().contiguous() if cam == "mei" else 0.0,
                 optimize_rig_rotation=optimize_rig_rotation)
        if optimize_rig_rotation:
            self.rig.copy_(rig)
    self.disps.clamp_(min=0.001)
