"""Host logic of the batched BA plan (no GPU needed: plan creation makes no CUDA call)."""

import ctypes

import pytest

from vipe_b200 import _lib
from vipe_b200 import workloads as W


def _ints(xs):
    return (ctypes.c_int * len(xs))(*xs)


def _plan(nf, ne, nk, t0, t1, ht=48, wd=64, ec=0, fc=0, group=3, adjoint=0):
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.vipe_slam_ba_batch_plan_create(len(nf), _ints(nf), _ints(ne), _ints(nk), _ints(t0), _ints(t1), ht, wd,
                                            ec, fc, group, adjoint, ctypes.byref(h))
    return rc, h


def test_plan_totals_and_workspace():
    b = W.make_ba_batch(5, seed=2, frames_range=(8, 14))
    rc, h = _plan(*b.sizes)
    assert rc == 0
    lib = _lib.load()
    tot = (ctypes.c_int64 * 5)()
    assert lib.vipe_slam_ba_batch_totals(h, tot) == 0
    assert list(tot)[:4] == [sum(b.num_frames), sum(b.num_edges), sum(b.num_kx), sum(f - 2 for f in b.num_frames)]
    ws = lib.vipe_slam_ba_batch_workspace_size(h)
    single = sum(lib.vipe_slam_ba_workspace_size(n, 48, 64, e, k, 2, n)
                 for n, e, k in zip(b.num_frames, b.num_edges, b.num_kx))
    assert ws > 0 and ws < 2 * single  # the batch needs about the sum of the graphs' workspaces
    lib.vipe_slam_ba_batch_plan_destroy(h)


@pytest.mark.parametrize(
    "bad, code",
    [
        (dict(t1=[8, 20]), _lib.VIPE_ERR_RANGE),  # t1 beyond num_frames
        (dict(t0=[2, 9], t1=[8, 9]), _lib.VIPE_ERR_RANGE),  # empty window
        (dict(nk=[6, 3]), _lib.VIPE_ERR_KX_MISMATCH),  # fewer depth rows than window poses
    ],
)
def test_plan_rejects_bad_graphs(bad, code):
    sz = dict(nf=[8, 10], ne=[26, 34], nk=[6, 8], t0=[2, 2], t1=[8, 10])
    sz.update(bad)
    rc, h = _plan(sz["nf"], sz["ne"], sz["nk"], sz["t0"], sz["t1"])
    assert rc == code and not h.value
    assert "graph 1" in _lib.load().vipe_last_error().decode()


def test_plan_rejects_empty_and_negative_chunks():
    rc, _ = _plan([], [], [], [], [])
    assert rc == 1
    rc, _ = _plan([8], [26], [6], [2], [8], ec=-1)
    assert rc == 1


def test_batch_generator_layout():
    b = W.make_ba_batch(3, seed=9, frames_range=(10, 12))
    t = b.tensors
    assert t["poses"].shape == (sum(b.num_frames), 7)
    assert t["targets"].shape == (sum(b.num_edges), 2, 48, 64)
    assert t["eta"].shape[0] == sum(b.num_kx)
    eo = 0
    for g in range(b.G):
        ii = t["ii"][eo:eo + b.num_edges[g]]
        jj = t["jj"][eo:eo + b.num_edges[g]]
        assert int(ii.max()) < b.num_frames[g] and int(jj.max()) < b.num_frames[g]  # local indices
        eo += b.num_edges[g]
    p = b.clip(1)
    assert p.poses.shape[0] == b.num_frames[1] and p.ii.shape[0] == b.num_edges[1]


def test_plan_groups():
    sz = ([8, 10], [26, 34], [6, 8], [2, 2], [8, 10])
    rc, h = _plan(*sz, group=4)
    assert rc == 0
    lib = _lib.load()
    tot = (ctypes.c_int64 * 5)()
    lib.vipe_slam_ba_batch_totals(h, tot)
    rc3, h3 = _plan(*sz, group=3)
    assert lib.vipe_slam_ba_batch_workspace_size(h) > lib.vipe_slam_ba_batch_workspace_size(h3)  # 7x7 blocks
    lib.vipe_slam_ba_batch_plan_destroy(h)
    lib.vipe_slam_ba_batch_plan_destroy(h3)
    assert _plan(*sz, group=5)[0] == _lib.VIPE_ERR_GROUP
    rc7, h7 = _plan(*sz, group=4, adjoint=1)  # Sim3 plans take the adjoint too
    assert rc7 == 0
    lib.vipe_slam_ba_batch_plan_destroy(h7)
    # Sim3 windows are limited to 109 poses (7 P + 1 unknowns in the staged Cholesky panel)
    assert _plan([120], [200], [118], [2], [120], group=4)[0] == _lib.VIPE_ERR_CAPACITY
