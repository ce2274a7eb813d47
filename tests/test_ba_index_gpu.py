"""Device-built BA graph index vs the reference's host index construction, bit for bit.

The reference builds its index on the host (csrc/slam_ext/geom_kernels.cu):
  * kx, kk_exp = _unique(cat(arange(t0, t1), ii), sorted, inverse)  (:1649-1656);
  * the CSR that accum_cuda(., ii, kx) gathers rows with (:1043-1089, used at :1766-1785);
  * the pose pairs that receive a Schur block, from schur_block's enumeration (:1440-1468).
oracle/ba_oracle.cpp restates those loops (build_index, oracle_accum_csr,
schur_pairs).  vipe_b200 builds the same information on the GPU in one
kernel (ba_index_kernel); vipe_slam_ba_index_debug copies it out.  Every list
is compared with assert_array_equal: integer work, no tolerance.
"""

import ctypes

import numpy as np
import pytest
import torch

import oracle.ba as ob

pytestmark = pytest.mark.gpu


def _device_index(ii, jj, num_frames, t0, t1):
    from vipe_b200 import _lib

    lib = _lib.load()
    ii_np = np.asarray(ii, dtype=np.int64)
    E = ii_np.shape[0]
    K = len(np.unique(np.concatenate([np.arange(t0, t1), ii_np])))
    P = t1 - t0
    dii = torch.as_tensor(ii_np).cuda()
    djj = torch.as_tensor(np.asarray(jj, dtype=np.int64)).cuda()
    ws_bytes = lib.vipe_slam_ba_workspace_size(num_frames, 1, 1, E, K, t0, t1)
    ws = torch.empty(max(int(ws_bytes), 16), dtype=torch.uint8, device="cuda")
    kx = np.zeros(K, dtype=np.int64)
    kk = np.zeros(P + E, dtype=np.int64)
    cap = P * P
    pairs = np.zeros(2 * cap, dtype=np.int32)
    npairs = ctypes.c_int(0)
    cptr = np.zeros(K + 1, dtype=np.int64)
    cidx = np.zeros(max(E, 1), dtype=np.int64)
    rc = lib.vipe_slam_ba_index_debug(
        dii.data_ptr(), djj.data_ptr(), num_frames, E, K, t0, t1, kx.ctypes.data, kk.ctypes.data,
        pairs.ctypes.data, cap, ctypes.addressof(npairs), cptr.ctypes.data, cidx.ctypes.data, ws.data_ptr(),
        int(ws_bytes), torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, "vipe_slam_ba_index_debug")
    n = npairs.value
    return kx, kk, pairs[:2 * n].reshape(n, 2), cptr, cidx[:E]


def _check(ii, jj, num_frames, t0, t1):
    kx, kk, pairs, cptr, cidx = _device_index(ii, jj, num_frames, t0, t1)
    wkx, wkk = ob.index(ii, jj, t0, t1)
    np.testing.assert_array_equal(kx, wkx)
    np.testing.assert_array_equal(kk, wkk)
    wptr, widx = ob.accum_csr(ii, jj, t0, t1)
    np.testing.assert_array_equal(cptr, wptr)
    np.testing.assert_array_equal(cidx, widx)
    pi, pj, _ = ob.schur_pairs(ii, jj, t0, t1)
    want = np.unique(np.stack([pi, pj], 1), axis=0) if len(pi) else np.zeros((0, 2), np.int64)
    np.testing.assert_array_equal(pairs.astype(np.int64), want)
    return len(kx), len(pairs)


def test_index_reference_four_frame_case():
    # tests/test_slam_ext_ba_extended.py:_make_ba_inputs: 4 frames, window [1, 4)
    _check([1, 2, 2, 3, 3], [0, 0, 1, 1, 2], 4, 1, 4)


@pytest.mark.parametrize("cfg", ["ba_config0", "ba_config1"])
def test_index_configs(cfg):
    from vipe_b200 import workloads as W

    p = getattr(W, cfg)()
    K, npairs = _check(p.ii.numpy(), p.jj.numpy(), p.disps.shape[0], p.t0, p.t1)
    assert K == p.eta.shape[0] and npairs > 0


def test_index_stereo_duplicate_self_and_outside_window_edges():
    """Self edges (ii == jj: the reference's stereo rule), duplicated edges, edges whose both ends
    lie before the window (their depth frame is still optimised) and edges into fixed poses."""
    ii = [0, 1, 2, 3, 3, 4, 4, 5, 6, 7, 7, 8, 9, 0, 1, 9, 2, 5]
    jj = [1, 0, 3, 3, 4, 5, 5, 4, 6, 8, 2, 7, 0, 9, 0, 9, 1, 2]
    _check(ii, jj, 10, 2, 9)


def test_index_empty_window_neighbours_and_last_frame():
    """Window ending at the last frame, depth frames that only appear through edges."""
    ii = [5, 6, 7, 11, 11, 0]
    jj = [6, 5, 11, 7, 10, 11]
    _check(ii, jj, 12, 6, 12)


def test_index_batch_clips():
    """16 clips of the uneven batch workload (|i-j| <= 3 plus Poisson(4) loop pairs), each
    indexed as its own graph."""
    from vipe_b200 import workloads as W

    b = W.make_ba_batch(16, seed=1004, ht=8, wd=8)
    t = b.tensors
    eo = 0
    for g in range(b.G):
        e = b.num_edges[g]
        ii = t["ii"][eo:eo + e].numpy()
        jj = t["jj"][eo:eo + e].numpy()
        eo += e
        K, _ = _check(ii, jj, b.num_frames[g], b.t0[g], b.t1[g])
        assert K == b.num_kx[g]
