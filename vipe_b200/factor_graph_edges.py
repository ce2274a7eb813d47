"""Factor-graph edge construction on the GPU (the host loops of the reference's
FactorGraph.add_proximity_factors, vipe/slam/components/factor_graph.py:409-486).

proximity_edges(d, ...) runs the candidate suppression, the neighbourhood edges and the
greedy distance-ordered NMS in one kernel (vipe_slam_proximity_edges) and returns the same
(ii, jj) lists, in the same order, as the reference's loops; one synchronisation reads the
edge count (the reference synchronises once per candidate).

add_proximity_factors is a drop-in for the reference method with the same signature: it
computes the candidate distances the reference's way (self.buffer.frame_distance_dense_disp,
which calls slam_ext.frame_distance) and hands the edges to self.add_factors, so a
FactorGraph can take it as its method:

    FactorGraph.add_proximity_factors = vipe_b200.factor_graph_edges.add_proximity_factors
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib


def proximity_edges(d, ii_exist, jj_exist, t0, t1, t, rad=2, nms=2, thresh=16.0, max_factors=48, cross_view=False):
    """d: ((t - t0) * (t - t1),) float32 CUDA distances of candidates (i, j), i in [t0, t),
    j in [t1, t), row-major; ii_exist, jj_exist: the graph's active then inactive edges.
    Returns (ii, jj) int64 CUDA tensors."""
    _lib.require_cuda("d", d)
    dev = d.device
    d = d.reshape(-1).float().contiguous()
    if t1 < 0 or t0 < t1 or t <= t0:
        raise RuntimeError("proximity_edges: needs 0 <= t1 <= t0 < t")
    if d.numel() != (t - t0) * (t - t1):
        raise RuntimeError("proximity_edges: d must hold (t - t0) * (t - t1) candidate distances")
    ie = torch.as_tensor(ii_exist, dtype=torch.int64, device=dev).reshape(-1).contiguous()
    je = torch.as_tensor(jj_exist, dtype=torch.int64, device=dev).reshape(-1).contiguous()
    if ie.numel() != je.numel():
        raise RuntimeError("proximity_edges: ii_exist and jj_exist differ in length")
    lib = _lib.load()
    cap = int(lib.vipe_slam_proximity_edges_capacity(t0, t1, t, rad, max_factors, int(bool(cross_view))))
    ws_bytes = int(lib.vipe_slam_proximity_edges_workspace_size(t0, t1, t))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    ii = torch.empty(cap, dtype=torch.int64, device=dev)
    jj = torch.empty(cap, dtype=torch.int64, device=dev)
    n = torch.zeros(1, dtype=torch.int32, device=dev)
    rc = lib.vipe_slam_proximity_edges(d.data_ptr(), ie.data_ptr() if ie.numel() else None,
                                       je.data_ptr() if je.numel() else None, int(ie.numel()), t0, t1, t, rad, nms,
                                       ctypes.c_float(thresh), max_factors, int(bool(cross_view)), ii.data_ptr(),
                                       jj.data_ptr(), cap, n.data_ptr(), ws.data_ptr(), ws_bytes, _lib.stream_of(d))
    _lib.check(rc, "proximity_edges")
    k = int(n.item())
    return ii[:k], jj[:k]


def add_proximity_factors(self, t0: int = 0, t1: int = 0, rad: int = 2, nms: int = 2, beta: float = 0.25,
                          thresh: float = 16.0, remove: bool = False):
    """FactorGraph.add_proximity_factors with the edge construction on the GPU (same
    arguments, same edges; reference factor_graph.py:409-486)."""
    assert t0 >= t1, "t0 should be a subset of t1"
    t = self.buffer.n_frames
    if t <= t0:
        return
    ix = torch.arange(t0, t, device=self.device)
    jx = torch.arange(t1, t, device=self.device)
    ii, jj = torch.meshgrid(ix, jx, indexing="ij")
    d = self.buffer.frame_distance_dense_disp(ii.reshape(-1), jj.reshape(-1), beta=beta).mean(-1)
    ie = torch.cat([self.ii, self.ii_inac]).to(d.device)
    je = torch.cat([self.jj, self.jj_inac]).to(d.device)
    ei, ej = proximity_edges(d, ie, je, t0, t1, t, rad=rad, nms=nms, thresh=thresh, max_factors=self.max_factors,
                             cross_view=bool(self.cross_view))
    if ei.numel() == 0:
        return
    self.add_factors(ei, ej, remove)
