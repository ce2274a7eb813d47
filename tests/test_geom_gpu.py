"""slam_ext geometry helpers on the GPU against the FP64 oracle (oracle/geom.py).

frame_distance, projmap, iproj at float32 tolerances; depth_filter counts are
compared exactly except at pixels whose depth test sits within float rounding
of the threshold.  Out-of-range indices give NaN (frame_distance, projmap)
instead of an out-of-bounds read.
"""

import numpy as np
import pytest
import torch

import oracle.geom as og
from vipe_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _slam():
    from vipe_b200.ext import slam_ext

    return slam_ext


def _problem():
    p = W.ba_small(n_frames=8, ht=12, wd=16, seed=21)
    return p


def test_projmap_and_iproj():
    p = _problem()
    s = _slam()
    ii = torch.tensor([0, 1, 2, 5, 3])
    jj = torch.tensor([1, 0, 4, 5, 2])
    coords, valid = s.projmap(p.poses.cuda(), p.disps.cuda(), p.intrinsics.cuda(), ii.cuda(), jj.cuda())
    wc, wv = og.projmap(p.poses.numpy(), p.disps.numpy(), p.intrinsics.numpy(), ii.numpy(), jj.numpy())
    np.testing.assert_allclose(coords.cpu().numpy(), wc, atol=2e-4, rtol=1e-5)
    np.testing.assert_array_equal(valid.cpu().numpy(), wv)
    pts = s.iproj(p.poses.cuda(), p.disps.cuda(), p.intrinsics.cuda())
    np.testing.assert_allclose(pts.cpu().numpy(), og.iproj(p.poses.numpy(), p.disps.numpy(), p.intrinsics.numpy()),
                               rtol=1e-4, atol=1e-4)


def test_frame_distance():
    p = _problem()
    s = _slam()
    pi = torch.tensor([0, 1, 2, 3, 7, 0])
    pj = torch.tensor([1, 2, 4, 6, 0, 0])
    q = torch.zeros(6, dtype=torch.long)
    intr = p.intrinsics.view(1, 4)
    for beta in (0.7, 0.0, 1.0):
        d = s.frame_distance(p.poses.cuda(), p.disps.cuda(), intr.cuda(), pi.cuda(), pj.cuda(), q.cuda(), q.cuda(),
                             pi.cuda(), beta)
        want = og.frame_distance(p.poses.numpy(), p.disps.numpy(), intr.numpy(), pi.numpy(), pj.numpy(), q.numpy(),
                                 q.numpy(), pi.numpy(), beta)
        np.testing.assert_allclose(d.cpu().numpy(), want, rtol=1e-4, atol=1e-4)
    # out-of-range index -> NaN, others unaffected
    bad = pj.clone()
    bad[2] = 99
    d = s.frame_distance(p.poses.cuda(), p.disps.cuda(), intr.cuda(), pi.cuda(), bad.cuda(), q.cuda(), q.cuda(),
                         pi.cuda(), 0.7)
    assert torch.isnan(d[2]) and torch.isfinite(d[[0, 1, 3, 4, 5]]).all()


def test_depth_filter_counts():
    p = _problem()
    s = _slam()
    ix = torch.tensor([0, 3, 7])
    thresh = torch.tensor([0.3, 0.05, 1.0])
    c = s.depth_filter(p.poses.cuda(), p.disps.cuda(), p.intrinsics.cuda(), ix.cuda(), thresh.cuda())
    want = og.depth_filter(p.poses.numpy(), p.disps.numpy(), p.intrinsics.numpy(), ix.numpy(), thresh.numpy())
    got = c.cpu().numpy()
    assert got.shape == want.shape
    assert (np.abs(got - want) <= 1).all()  # at most one borderline neighbour per pixel
    assert (got == want).mean() > 0.99
