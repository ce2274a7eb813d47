"""Differentiable batched bundle adjustment (forward + hand-written adjoint).

    plan = BatchPlan(*sizes, ht, wd, device, adjoint=True)
    poses_out, disps_out = bundle_adjust(plan, poses, disps, targets, weights, eta, disps_sens,
                                         intrinsics, ii, jj, depth_active, iterations=2, lm=1e-4, ep=0.1)
    loss(poses_out, disps_out).backward()

The forward is the batched FP32 solve (vipe_slam_ba_batch_solve) run on copies
of poses/disps, recording the state entering every LM iteration, the factorised
reduced system and the pose step (no Jacobian is stored); the backward
is vipe_slam_ba_batch_backward: each LM step differentiated exactly (second
derivatives of the reprojection and the LM damping ep + lm*diag(S) included),
its linear solve differentiated implicitly by re-solving the same damped reduced
system with the incoming gradients, and the Jacobians recomputed from the
recorded states.  The reference has no BA
backward (its update operator is trained through a torch BA instead).

Gradient layout for poses follows lietorch (csrc/lietorch_ext/lietorch_gpu.cu:
85-98): the gradient with respect to a pose tensor (N, 7) is the left-tangent
gradient d loss / d eps of T -> Exp(eps) T in columns 0..5, column 6 zero — both
for the gradient flowing in (as lietorch's SE3 ops produce it) and for the one
returned.  Sim3 plans (group="sim3", poses (N, 8) [t q s]) use the same rule with the
tangent [tau phi sigma] in columns 0..6 and column 7 zero.  Gradients are returned for poses, disps, targets, weights, eta and
disps_sens; not for intrinsics, ii, jj or depth_active.
"""

from __future__ import annotations

import torch

from . import _lib
from .ba_batch import BatchPlan


class _BundleAdjust(torch.autograd.Function):
    @staticmethod
    def forward(ctx, plan, iterations, lm, ep, alpha, poses, disps, targets, weights, eta, disps_sens, intrinsics, ii,
                jj, depth_active):
        iterations = int(iterations)
        poses_out = poses.detach().clone().contiguous()
        disps_out = disps.detach().clone().contiguous()
        intr = intrinsics.detach().clone().contiguous()
        dev = poses.device
        tape = plan.make_tape(iterations)
        plan.solve(poses_out, disps_out, intr, disps_sens.detach(), targets.detach(), weights.detach(), eta.detach(),
                   ii, jj, depth_active.detach(), iterations, lm, ep, alpha=alpha, tape=tape)
        ctx.save_for_backward(*tape, targets.detach(), weights.detach(), eta.detach(), disps_sens.detach(),
                              intrinsics.detach(), ii, jj, depth_active.detach())
        ctx.plan = plan
        ctx.cfg = (iterations, float(lm), float(ep), float(alpha))
        return poses_out, disps_out

    @staticmethod
    def backward(ctx, g_poses, g_disps):
        tape_p, tape_d, tape_f, tape_x, targets, weights, eta, disps_sens, intrinsics, ii, jj, depth_active = (
            ctx.saved_tensors)
        plan = ctx.plan
        iterations, lm, ep, alpha = ctx.cfg
        dev = tape_p.device
        D = plan.dof
        gp = torch.zeros(plan.total_frames, D + 1, dtype=torch.float32, device=dev)
        gd = torch.zeros(plan.total_frames, plan.ht, plan.wd, dtype=torch.float32, device=dev)
        if g_poses is not None:
            gp.copy_(g_poses)
            gp[:, D] = 0.0
        if g_disps is not None:
            gd.copy_(g_disps)
        gt = torch.empty_like(targets)
        gw = torch.empty_like(weights)
        ge = torch.empty_like(eta)
        gs = torch.empty_like(disps_sens)
        status = torch.zeros(plan.G, dtype=torch.int32, device=dev)
        rc = _lib.load().vipe_slam_ba_batch_backward(
            plan._h, tape_p.data_ptr(), tape_d.data_ptr(), tape_f.data_ptr(), tape_x.data_ptr(),
            intrinsics.contiguous().data_ptr(), disps_sens.data_ptr(), targets.data_ptr(), weights.data_ptr(),
            eta.data_ptr(), ii.data_ptr(), jj.data_ptr(), depth_active.data_ptr(), iterations, lm, ep, alpha,
            gp.data_ptr(), gd.data_ptr(), gt.data_ptr(), gw.data_ptr(), ge.data_ptr(), gs.data_ptr(), status.data_ptr(),
            torch.cuda.current_stream(dev).cuda_stream,
        )
        _lib.check(rc, "bundle_adjust backward")
        ctx.status = status
        return (None, None, None, None, None, gp, gd, gt, gw, ge, gs, None, None, None, None)


def bundle_adjust(plan: BatchPlan, poses, disps, targets, weights, eta, disps_sens, intrinsics, ii, jj, depth_active,
                  iterations: int, lm: float, ep: float, alpha: float = 0.001):
    """Differentiable batched BA; returns (poses_out, disps_out) (inputs are not modified)."""
    if not plan.adjoint:
        raise RuntimeError("bundle_adjust needs a BatchPlan created with adjoint=True")
    return _BundleAdjust.apply(plan, iterations, lm, ep, alpha, poses, disps, targets, weights, eta, disps_sens,
                               intrinsics, ii, jj, depth_active)
