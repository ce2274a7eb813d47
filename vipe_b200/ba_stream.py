"""Host-resident batches streamed through the GPU: batched BA forward + adjoint
with the host<->device copies overlapped with the solves.

A caller whose clips live in (pinned) host memory pays, per step, the copy of
every input to the GPU and of every result back.  Issued in sequence around one
batched solve those copies add to it; here the batch is cut into ``parts``
groups of consecutive clips (balanced by edge count), each with its own bound
plan, tape, device buffers and CUDA stream, and one ``step`` enqueues for every
part, on its own stream: host->device copies of its slice, the forward solve
recording its tape, the hand-written backward, and device->host copies of its
outputs.  The copy engines move one part while the SMs solve another, so a step
costs about the largest of (copies in, solves, copies out) plus one part's copies.

    runner = StreamedBundleAdjust(sizes, ht, wd, "cuda", parts=8, iterations=4, lm=1e-4, ep=0.1)
    host_out = runner.host_outputs()                  # pinned result buffers
    runner.step(host_batch, host_grad_poses, host_grad_disps, host_out)
    torch.cuda.current_stream().synchronize()

Per-graph arithmetic is the batched plan's: each graph's result does not depend
on which other graphs share its launch, so a streamed step returns the same
values as one plan over the whole batch with the same pixel chunking.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from .ba_batch import BATCH_KEYS, BatchPlan

# outputs copied back per step: the solved state and every input gradient
OUTPUT_KEYS = ("poses", "disps", "grad_poses", "grad_disps", "grad_targets", "grad_weights", "grad_eta",
               "grad_disps_sens")


def split_clips(num_edges, parts: int, taper: float = 1.0) -> list[tuple[int, int]]:
    """Cuts graphs 0..G-1 into at most ``parts`` non-empty ranges of consecutive
    graphs with edge totals (each graph's edges + 1, so edge-free graphs still
    count) in proportion to the part weights: 1 for every part, ``taper`` for the
    first and the last of three or more.  A small first part starts the solves
    sooner (its copy-in is the only one nothing overlaps) and a small last part
    ends the step sooner (likewise its copy-out)."""
    G = len(num_edges)
    parts = max(1, min(int(parts), G))
    w = [int(e) + 1 for e in num_edges]
    total = sum(w)
    pw = [1.0] * parts
    if parts >= 3:
        pw[0] = pw[-1] = float(taper)
    bounds, run = [], 0.0
    for x in pw:
        run += x
        bounds.append(run / sum(pw))  # cumulative share ending each part
    cuts, acc, k = [0], 0, 1
    for g in range(G):
        acc += w[g]
        left = G - (g + 1)  # graphs after this one; every remaining part needs one
        if k < parts and left >= parts - k and (acc >= total * bounds[k - 1] or left == parts - k):
            cuts.append(g + 1)
            k += 1
    cuts.append(G)
    return [(cuts[i], cuts[i + 1]) for i in range(len(cuts) - 1) if cuts[i + 1] > cuts[i]]


@dataclass
class _Part:
    g: tuple[int, int]   # graph range
    f: tuple[int, int]   # frame rows
    e: tuple[int, int]   # edge rows
    k: tuple[int, int]   # eta rows
    plan: BatchPlan
    stream: torch.cuda.Stream
    dev: dict
    grads: dict
    tape: tuple
    out: tuple
    status: torch.Tensor
    done: torch.cuda.Event


class StreamedBundleAdjust:
    """Batched BA forward + adjoint over host-resident inputs, copies overlapped with compute."""

    def __init__(self, sizes, ht: int, wd: int, device, parts: int = 8, iterations: int = 4, lm: float = 1e-4,
                 ep: float = 0.1, alpha: float = 0.001, edge_chunks: int = 0, frame_chunks: int = 0,
                 group: str = "se3", adjoint: bool = True, taper: float = 0.25):
        num_frames, num_edges, num_kx, t0, t1 = (list(map(int, x)) for x in sizes)
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.ht, self.wd = int(ht), int(wd)
        self.iterations, self.lm, self.ep, self.alpha = int(iterations), float(lm), float(ep), float(alpha)
        self.G = len(num_frames)
        self.total_frames, self.total_edges, self.total_kx = sum(num_frames), sum(num_edges), sum(num_kx)
        self.dof = 7 if group == "sim3" else 6
        self.adjoint = bool(adjoint)
        self.parts: list[_Part] = []
        HW = (self.ht, self.wd)
        f0 = e0 = k0 = 0
        for ga, gb in split_clips(num_edges, parts, taper):
            nf, ne, nk = sum(num_frames[ga:gb]), sum(num_edges[ga:gb]), sum(num_kx[ga:gb])
            plan = BatchPlan(num_frames[ga:gb], num_edges[ga:gb], num_kx[ga:gb], t0[ga:gb], t1[ga:gb], self.ht,
                             self.wd, self.device, edge_chunks=edge_chunks, frame_chunks=frame_chunks,
                             adjoint=self.adjoint, group=group)
            dev = self.device
            f32 = dict(dtype=torch.float32, device=dev)
            d = {
                "poses": torch.empty(nf, self.dof + 1, **f32),
                "disps": torch.empty(nf, *HW, **f32),
                "intrinsics": torch.empty(gb - ga, 4, **f32),
                "disps_sens": torch.empty(nf, *HW, **f32),
                "targets": torch.empty(ne, 2, *HW, **f32),
                "weights": torch.empty(ne, 2, *HW, **f32),
                "eta": torch.empty(nk, *HW, **f32),
                "ii": torch.empty(ne, dtype=torch.int64, device=dev),
                "jj": torch.empty(ne, dtype=torch.int64, device=dev),
                "depth_active": torch.empty(nf, **f32),
            }
            grads = {
                "grad_poses": torch.empty(nf, self.dof + 1, **f32),
                "grad_disps": torch.empty(nf, *HW, **f32),
                "grad_targets": torch.empty(ne, 2, *HW, **f32),
                "grad_weights": torch.empty(ne, 2, *HW, **f32),
                "grad_eta": torch.empty(nk, *HW, **f32),
                "grad_disps_sens": torch.empty(nf, *HW, **f32),
            } if self.adjoint else {}
            self.parts.append(_Part(g=(ga, gb), f=(f0, f0 + nf), e=(e0, e0 + ne), k=(k0, k0 + nk), plan=plan,
                                    stream=torch.cuda.Stream(dev), dev=d, grads=grads,
                                    tape=plan.make_tape(self.iterations) if self.adjoint else None,
                                    out=plan.outputs(self.iterations),
                                    status=torch.zeros(gb - ga, dtype=torch.int32, device=dev),
                                    done=torch.cuda.Event()))
            f0, e0, k0 = f0 + nf, e0 + ne, k0 + nk

    def host_outputs(self) -> dict:
        """Pinned host buffers for every output of a step."""
        HW = (self.ht, self.wd)
        pin = dict(dtype=torch.float32, pin_memory=True)
        F, E, K = self.total_frames, self.total_edges, self.total_kx
        if not self.adjoint:
            return {"poses": torch.empty(F, self.dof + 1, **pin), "disps": torch.empty(F, *HW, **pin)}
        return {
            "poses": torch.empty(F, self.dof + 1, **pin),
            "disps": torch.empty(F, *HW, **pin),
            "grad_poses": torch.empty(F, self.dof + 1, **pin),
            "grad_disps": torch.empty(F, *HW, **pin),
            "grad_targets": torch.empty(E, 2, *HW, **pin),
            "grad_weights": torch.empty(E, 2, *HW, **pin),
            "grad_eta": torch.empty(K, *HW, **pin),
            "grad_disps_sens": torch.empty(F, *HW, **pin),
        }

    def _rows(self, part: _Part, key: str):
        if key in ("targets", "weights", "ii", "jj", "grad_targets", "grad_weights"):
            return part.e
        if key in ("eta", "grad_eta"):
            return part.k
        if key == "intrinsics":
            return part.g
        return part.f

    def step(self, host: dict, host_grad_poses: torch.Tensor | None, host_grad_disps: torch.Tensor | None,
             host_out: dict, stream: torch.cuda.Stream | None = None) -> None:
        """Enqueues one forward (+ backward) over the batch held in pinned host tensors.

        ``host`` holds the batched inputs (BATCH_KEYS, concatenated layout),
        host_grad_poses / host_grad_disps the incoming gradients of the solved
        poses and depths (None for a forward-only runner); ``host_out`` (from
        host_outputs) receives the solved state and, with the adjoint, every
        input gradient.  Work starts after what is already queued
        on ``stream`` (default: the current stream) and that stream waits for all
        of it, so events recorded there bracket the whole step."""
        caller = stream if stream is not None else torch.cuda.current_stream(self.device)
        start = torch.cuda.Event()
        start.record(caller)
        for part in self.parts:
            part.stream.wait_event(start)
            with torch.cuda.stream(part.stream):
                for key in BATCH_KEYS:
                    a, b = self._rows(part, key)
                    part.dev[key].copy_(host[key][a:b], non_blocking=True)
                fa, fb = part.f
                d, gr = part.dev, part.grads
                # the solve and the backward OR their per-graph words in: clear last step's
                part.out[3].zero_()
                part.status.zero_()
                if self.adjoint:
                    gr["grad_poses"].copy_(host_grad_poses[fa:fb], non_blocking=True)
                    gr["grad_disps"].copy_(host_grad_disps[fa:fb], non_blocking=True)
                part.plan.solve(**d, iterations=self.iterations, lm=self.lm, ep=self.ep, alpha=self.alpha,
                                out=part.out, check=False, tape=part.tape)
                if self.adjoint:
                    part.plan.backward(part.tape, d["intrinsics"], d["disps_sens"], d["targets"], d["weights"],
                                       d["eta"], d["ii"], d["jj"], d["depth_active"], self.iterations, self.lm, self.ep,
                                       self.alpha, gr["grad_poses"], gr["grad_disps"], gr["grad_targets"],
                                       gr["grad_weights"], gr["grad_eta"], gr["grad_disps_sens"], part.status)
                for key in host_out:
                    a, b = self._rows(part, key)
                    src = d[key] if key in d else gr[key]
                    host_out[key][a:b].copy_(src, non_blocking=True)
                part.done.record(part.stream)
            caller.wait_event(part.done)

    def status(self) -> torch.Tensor:
        """Per-graph device status words of the last step (solve | backward), in batch order."""
        return torch.cat([p.out[3] | p.status for p in self.parts])

    def h2d_bytes(self, host: dict) -> int:
        grads = self.total_frames * (self.dof + 1) * 4 + self.total_frames * self.ht * self.wd * 4
        return sum(host[k].numel() * host[k].element_size() for k in BATCH_KEYS) + (grads if self.adjoint else 0)

    def d2h_bytes(self, host_out: dict) -> int:
        return sum(v.numel() * v.element_size() for v in host_out.values())
