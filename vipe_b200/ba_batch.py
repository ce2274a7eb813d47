"""Batched dense bundle adjustment: many clips' factor graphs in one solve.

The reference solves one keyframe graph per ``slam_ext.ba_extended`` call
(vipe csrc/slam_ext/geom_kernels.cu:1626-1847).  Here graphs of uneven frame
and edge counts are laid side by side (every tensor concatenated along its
leading axis, edge indices local to their graph) and each phase of the LM step
is one launch over all of them: per-edge terms, per-frame Schur products,
assembly, one FP64 Cholesky CTA per graph, back-substitution and retraction.

    plan = BatchPlan([g.num_frames ...], [E ...], [K ...], [t0 ...], [t1 ...], ht, wd, device)
    batch = concat_problems(problems)          # dict of concatenated tensors
    out = plan.solve(**batch, iterations=4, lm=1e-4, ep=0.1)
    graph = plan.capture(batch, iterations=4, lm=1e-4, ep=0.1)   # CUDA graph of the LM loop
    graph.replay()

``autotune`` picks the pixel chunking of the two linearisation kernels by
timing the candidates on the batch itself.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _lib


def _ints(xs) -> ctypes.Array:
    xs = [int(x) for x in xs]
    return (ctypes.c_int * len(xs))(*xs)


class BatchPlan:
    """A bound plan: graph table uploaded into a device workspace on `device`."""

    def __init__(self, num_frames, num_edges, num_kx, t0, t1, ht: int, wd: int, device, edge_chunks: int = 0,
                 frame_chunks: int = 0, adjoint: bool = False, group: str = "se3"):
        lib = _lib.load()
        self.G = len(num_frames)
        if not (len(num_edges) == len(num_kx) == len(t0) == len(t1) == self.G) or self.G == 0:
            raise RuntimeError("BatchPlan: per-graph size lists must be non-empty and of equal length")
        self.ht, self.wd = int(ht), int(wd)
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.sizes = (tuple(map(int, num_frames)), tuple(map(int, num_edges)), tuple(map(int, num_kx)),
                      tuple(map(int, t0)), tuple(map(int, t1)))
        self.edge_chunks, self.frame_chunks = int(edge_chunks), int(frame_chunks)
        self.adjoint = bool(adjoint)
        if group not in ("se3", "sim3"):
            raise RuntimeError("BatchPlan: group must be 'se3' or 'sim3'")
        self.group = group
        self.dof = 7 if group == "sim3" else 6
        h = ctypes.c_void_p()
        rc = lib.vipe_slam_ba_batch_plan_create(self.G, _ints(num_frames), _ints(num_edges), _ints(num_kx), _ints(t0),
                                                _ints(t1), self.ht, self.wd, self.edge_chunks, self.frame_chunks,
                                                3 if group == "se3" else 4, int(self.adjoint), ctypes.byref(h))
        _lib.check(rc, "BatchPlan")
        self._h = h
        tot = (ctypes.c_int64 * 5)()
        _lib.check(lib.vipe_slam_ba_batch_totals(h, tot), "BatchPlan")
        self.total_frames, self.total_edges, self.total_kx, self.total_poses, self.factor_tape_doubles = (
            int(x) for x in tot)
        nbytes = int(lib.vipe_slam_ba_batch_workspace_size(h))
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            rc = lib.vipe_slam_ba_batch_bind(h, self.workspace.data_ptr(), nbytes,
                                             torch.cuda.current_stream(self.device).cuda_stream)
        _lib.check(rc, "BatchPlan.bind")

    @classmethod
    def for_problems(cls, problems, device, **kw) -> "BatchPlan":
        return cls([p.disps.shape[0] for p in problems], [p.num_edges for p in problems],
                   [p.eta.shape[0] for p in problems], [p.t0 for p in problems], [p.t1 for p in problems],
                   problems[0].disps.shape[1], problems[0].disps.shape[2], device, **kw)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().vipe_slam_ba_batch_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    def _check(self, poses, disps, intrinsics, disps_sens, targets, weights, eta, ii, jj, depth_active):
        HW = (self.ht, self.wd)
        want = {
            "poses": (poses, (self.total_frames, self.dof + 1), torch.float32),
            "disps": (disps, (self.total_frames, *HW), torch.float32),
            "intrinsics": (intrinsics, (self.G, 4), torch.float32),
            "disps_sens": (disps_sens, (self.total_frames, *HW), torch.float32),
            "targets": (targets, (self.total_edges, 2, *HW), torch.float32),
            "weights": (weights, (self.total_edges, 2, *HW), torch.float32),
            "eta": (eta, (self.total_kx, *HW), torch.float32),
            "ii": (ii, (self.total_edges,), torch.int64),
            "jj": (jj, (self.total_edges,), torch.int64),
            "depth_active": (depth_active, (self.total_frames,), torch.float32),
        }
        for name, (t, shape, dt) in want.items():
            _lib.require_cuda(name, t)
            _lib.require_contiguous(name, t)
            _lib.require_dtype(name, t, dt)
            if tuple(t.shape) != shape:
                raise RuntimeError(f"BatchPlan.solve: {name} has shape {tuple(t.shape)}, the plan expects {shape}")
            if t.device != self.device:
                raise RuntimeError(f"BatchPlan.solve: {name} is on {t.device}, the plan on {self.device}")

    def make_tape(self, iterations: int):
        """Buffers of the record the backward pass reads: per iteration the state
        entering it (poses, disps), the factorised reduced system with the per-pixel (Q, w)
        of the depth elimination, and the pose step."""
        dev, it = self.device, int(iterations)
        return (torch.empty(it, self.total_frames, self.dof + 1, dtype=torch.float32, device=dev),
                torch.empty(it, self.total_frames, self.ht, self.wd, dtype=torch.float32, device=dev),
                torch.empty(it, max(1, self.factor_tape_doubles), dtype=torch.float64, device=dev),
                torch.empty(it, max(1, self.total_poses), self.dof, dtype=torch.float32, device=dev))

    def outputs(self, iterations: int, motion_only: bool = False, compute_energy: bool = False):
        dev = self.device
        dx = torch.zeros(self.total_poses, self.dof, dtype=torch.float32, device=dev)
        dz = None if motion_only else torch.empty(self.total_kx, self.ht * self.wd, dtype=torch.float32, device=dev)
        energy = torch.zeros(self.G, iterations if compute_energy else 0, dtype=torch.float32, device=dev)
        status = torch.zeros(self.G, dtype=torch.int32, device=dev)
        return dx, dz, energy, status

    def solve(self, poses, disps, intrinsics, disps_sens, targets, weights, eta, ii, jj, depth_active, iterations,
              lm, ep, motion_only=False, alpha=0.001, optimize_intrinsics=False, intrinsics_lm=1e-6,
              intrinsics_ep=1e-6, intrinsics_scale=1.0, compute_energy=False, out=None, check=True, tape=None):
        """LM iterations on every graph; poses/disps/intrinsics are updated in place.

        Returns (dx, dz, energy, status): dx (sum P, 6 or 7), dz (sum K, H*W) or None,
        energy (G, iterations) or (G, 0), status (G,) int32 device words
        (0, a vipe_status error, or VIPE_WARN_SOLVER when that graph's Cholesky
        failed and its dx is 0).  ``out`` reuses preallocated outputs (for
        CUDA-graph capture; the solve ORs its words into ``out``'s status, so zero
        it between solves that should report separately); ``check`` validates
        shapes on the host; ``tape``
        (from make_tape) receives the record the backward pass reads.
        """
        if check:
            self._check(poses, disps, intrinsics, disps_sens, targets, weights, eta, ii, jj, depth_active)
        iterations = int(iterations)
        if out is None:
            out = self.outputs(iterations, motion_only, compute_energy)
        dx, dz, energy, status = out
        rc = _lib.load().vipe_slam_ba_batch_solve(
            self._h, poses.data_ptr(), disps.data_ptr(), intrinsics.data_ptr(), disps_sens.data_ptr(),
            targets.data_ptr(), weights.data_ptr(), eta.data_ptr(), ii.data_ptr(), jj.data_ptr(),
            depth_active.data_ptr(), iterations, float(lm), float(ep), int(bool(motion_only)), float(alpha),
            int(bool(optimize_intrinsics)), float(intrinsics_lm), float(intrinsics_ep), float(intrinsics_scale),
            int(bool(compute_energy)), dx.data_ptr(), _lib.ptr(dz), energy.data_ptr() if compute_energy else None,
            status.data_ptr(), *([None] * 4 if tape is None else [t.data_ptr() for t in tape]),
            torch.cuda.current_stream(self.device).cuda_stream,
        )
        _lib.check(rc, "BatchPlan.solve")
        return dx, dz, energy, status

    def backward(self, tape, intrinsics, disps_sens, targets, weights, eta, ii, jj, depth_active, iterations, lm, ep,
                 alpha, grad_poses, grad_disps, grad_targets, grad_weights, grad_eta, grad_disps_sens, status):
        """Hand-written adjoint of the solve that filled ``tape`` (plan created with adjoint=True).

        grad_poses (frames, dof+1) and grad_disps (frames, H, W) hold the incoming
        gradients of the solve's outputs and receive those of its input poses and
        depths; grad_targets, grad_weights, grad_eta, grad_disps_sens are written;
        status (G,) int32 receives per-graph device status.  Only enqueues work on
        the current stream (no allocation, copy or synchronisation)."""
        rc = _lib.load().vipe_slam_ba_batch_backward(
            self._h, *[t.data_ptr() for t in tape], intrinsics.data_ptr(), disps_sens.data_ptr(), targets.data_ptr(),
            weights.data_ptr(), eta.data_ptr(), ii.data_ptr(), jj.data_ptr(), depth_active.data_ptr(), int(iterations),
            float(lm), float(ep), float(alpha), grad_poses.data_ptr(), grad_disps.data_ptr(), grad_targets.data_ptr(),
            grad_weights.data_ptr(), grad_eta.data_ptr(), grad_disps_sens.data_ptr(), status.data_ptr(),
            torch.cuda.current_stream(self.device).cuda_stream)
        _lib.check(rc, "BatchPlan.backward")

    def capture(self, batch: dict, iterations: int, lm: float, ep: float, **kw) -> "CapturedSolve":
        """Captures the whole solve (index build + LM loop) on `batch`'s tensors as a CUDA graph."""
        return CapturedSolve(self, batch, iterations, lm, ep, **kw)


class CapturedSolve:
    """CUDA graph of one batched solve over fixed (static) tensors.

    replay() re-runs the solve on whatever the static tensors hold; copy new
    inputs into ``batch`` tensors first (poses/disps/intrinsics are updated in
    place by every replay)."""

    def __init__(self, plan: BatchPlan, batch: dict, iterations: int, lm: float, ep: float, **kw):
        self.plan, self.batch = plan, batch
        self.out = plan.outputs(int(iterations), kw.get("motion_only", False), kw.get("compute_energy", False))
        plan._check(**{k: batch[k] for k in BATCH_KEYS})
        args = dict(batch)
        self.graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(plan.device)
        side.wait_stream(torch.cuda.current_stream(plan.device))
        with torch.cuda.stream(side):
            with torch.cuda.graph(self.graph, stream=side):
                plan.solve(**{k: args[k] for k in BATCH_KEYS}, iterations=iterations, lm=lm, ep=ep, out=self.out,
                           check=False, **kw)
        torch.cuda.current_stream(plan.device).wait_stream(side)

    def replay(self):
        self.graph.replay()
        return self.out


BATCH_KEYS = ("poses", "disps", "intrinsics", "disps_sens", "targets", "weights", "eta", "ii", "jj", "depth_active")


def concat_problems(problems, device=None) -> dict:
    """Concatenates BAProblem-like objects into the batched layout (edge indices stay local)."""
    def cat(name):
        ts = [getattr(p, name) for p in problems]
        t = torch.cat([x.reshape(1, -1) if name == "intrinsics" else x for x in ts], 0).contiguous()
        return t if device is None else t.to(device)

    return {k: cat(k) for k in BATCH_KEYS}


def split_rows(t: torch.Tensor, counts) -> list[torch.Tensor]:
    """Splits a concatenated tensor back into per-graph pieces."""
    return list(torch.split(t, [int(c) for c in counts], 0))


# ---------------------------------------------------------------- autotuner

@dataclass
class TuneResult:
    edge_chunks: int
    frame_chunks: int
    ms: float
    table: list


_TUNE_CACHE: dict = {}

CANDIDATES = ((1, 1), (2, 1), (1, 2), (2, 2), (3, 2), (3, 4))


def autotune(plan_sizes: tuple, ht: int, wd: int, batch: dict, iterations: int, lm: float, ep: float, device,
             candidates=CANDIDATES, reps: int = 3, group: str = "se3", **kw) -> TuneResult:
    """Times each (edge_chunks, frame_chunks) candidate on copies of `batch` and returns the fastest.

    plan_sizes = (num_frames, num_edges, num_kx, t0, t1) lists.  Results are
    cached per (sizes, ht, wd, iterations, motion_only)."""
    key = (tuple(tuple(x) for x in plan_sizes), ht, wd, int(iterations), bool(kw.get("motion_only", False)), group)
    if key in _TUNE_CACHE:
        return _TUNE_CACHE[key]
    mutable = ("poses", "disps", "intrinsics")
    work = {k: (v.clone() if k in mutable else v) for k, v in batch.items()}
    table = []
    for ec, fc in candidates:
        plan = BatchPlan(*plan_sizes, ht, wd, device, edge_chunks=ec, frame_chunks=fc, group=group)
        out = plan.outputs(iterations, kw.get("motion_only", False), kw.get("compute_energy", False))
        times = []
        for r in range(reps + 1):
            for k in mutable:
                work[k].copy_(batch[k])
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            plan.solve(**work, iterations=iterations, lm=lm, ep=ep, out=out, check=(r == 0), **kw)
            b.record()
            b.synchronize()
            if r > 0:
                times.append(a.elapsed_time(b))
        table.append((ec, fc, min(times)))
        del plan
    best = min(table, key=lambda x: x[2])
    res = TuneResult(best[0], best[1], best[2], table)
    _TUNE_CACHE[key] = res
    return res
