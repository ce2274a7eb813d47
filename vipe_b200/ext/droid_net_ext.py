"""droid_net_ext — drop-in for the reference's ``vipe.ext.droid_net_ext`` pybind module.

Reference bindings: vipe csrc/droid_net_ext/droid.cpp:75-81.  Same function
names, positional arguments and list returns.  Lookups accumulate in FP32 and
write each output once (the reference accumulates in the volume dtype).
``altcorr_backward`` returns a zero coords gradient like the reference unless
``exact_coords_grad=True`` is passed (then the derivative of the bilinear
lookup is returned).  ``corr_index_coords_backward`` (not in the reference) is
the same derivative for the materialised-volume lookup, and
``altcorr_index_backward`` (not in the reference either) the adjoint of the
indexed lookup.
"""

from __future__ import annotations

import ctypes

import torch

from .. import _lib


def _check(name, t):
    _lib.require_cuda(name, t)
    _lib.require_contiguous(name, t)


def corr_index_forward(volume, coords, radius):
    """volume (B, h1, w1, h2, w2), coords (B, 2, h1, w1) f32 -> [corr (B, 2r+1, 2r+1, h1, w1)]."""
    _check("volume", volume)
    _check("coords", coords)
    _lib.require_dtype("coords", coords, torch.float32)
    B, h1, w1, h2, w2 = volume.shape
    rd = 2 * int(radius) + 1
    corr = torch.empty(B, rd, rd, h1, w1, dtype=volume.dtype, device=volume.device)
    rc = _lib.load().vipe_corr_index_forward(_lib.DTYPE_CODE[volume.dtype], volume.data_ptr(), coords.data_ptr(), B,
                                             h1, w1, h2, w2, int(radius), corr.data_ptr(), _lib.stream_of(volume))
    _lib.check(rc, "droid_net_ext.corr_index_forward")
    return [corr]


def corr_index_backward(volume, coords, corr_grad, radius):
    """-> [volume_grad (B, h1, w1, h2, w2)]."""
    _check("volume", volume)
    _check("coords", coords)
    _check("corr_grad", corr_grad)
    B, h1, w1, h2, w2 = volume.shape
    if corr_grad.dtype != volume.dtype:
        raise RuntimeError("corr_grad must have the volume's dtype")
    vg = torch.empty_like(volume)
    rc = _lib.load().vipe_corr_index_backward(_lib.DTYPE_CODE[volume.dtype], coords.data_ptr(), corr_grad.data_ptr(),
                                              B, h1, w1, h2, w2, int(radius), vg.data_ptr(), _lib.stream_of(volume))
    _lib.check(rc, "droid_net_ext.corr_index_backward")
    return [vg]


def corr_index_coords_backward(volume, coords, corr_grad, radius):
    """-> [coords_grad (B, 2, h1, w1) f32]: exact derivative of corr_index_forward in coords."""
    _check("volume", volume)
    _check("coords", coords)
    _check("corr_grad", corr_grad)
    _lib.require_dtype("coords", coords, torch.float32)
    B, h1, w1, h2, w2 = volume.shape
    if corr_grad.dtype != volume.dtype:
        raise RuntimeError("corr_grad must have the volume's dtype")
    cg = torch.empty(B, 2, h1, w1, dtype=torch.float32, device=volume.device)
    rc = _lib.load().vipe_corr_index_coords_backward(_lib.DTYPE_CODE[volume.dtype], volume.data_ptr(),
                                                     coords.data_ptr(), corr_grad.data_ptr(), B, h1, w1, h2, w2,
                                                     int(radius), cg.data_ptr(), _lib.stream_of(volume))
    _lib.check(rc, "droid_net_ext.corr_index_coords_backward")
    return [cg]


def altcorr_forward(fmap1, fmap2, coords, radius):
    """fmap1 (B,H1,W1,C), fmap2 (B,H2,W2,C), coords (B,S,H1,W1,2) -> [corr (B,S,(2r+1)^2,H1,W1)]."""
    for n, t in (("fmap1", fmap1), ("fmap2", fmap2), ("coords", coords)):
        _check(n, t)
    _lib.require_dtype("coords", coords, torch.float32)
    if fmap2.dtype != fmap1.dtype:
        raise RuntimeError("fmap1 and fmap2 must share a dtype")
    B, H1, W1, C = fmap1.shape
    _, H2, W2, _ = fmap2.shape
    S = coords.shape[1]
    rd = 2 * int(radius) + 1
    corr = torch.empty(B, S, rd * rd, H1, W1, dtype=fmap1.dtype, device=fmap1.device)
    rc = _lib.load().vipe_altcorr_forward(_lib.DTYPE_CODE[fmap1.dtype], fmap1.data_ptr(), fmap2.data_ptr(),
                                          coords.data_ptr(), B, S, H1, W1, H2, W2, C, int(radius), corr.data_ptr(),
                                          _lib.stream_of(fmap1))
    _lib.check(rc, "droid_net_ext.altcorr_forward")
    return [corr]


def altcorr_backward(fmap1, fmap2, coords, corr_grad, radius, exact_coords_grad=False):
    """float32 only (as the reference) -> [fmap1_grad, fmap2_grad, coords_grad]."""
    for n, t in (("fmap1", fmap1), ("fmap2", fmap2), ("coords", coords), ("corr_grad", corr_grad)):
        _check(n, t)
        _lib.require_dtype(n, t, torch.float32)
    B, H1, W1, C = fmap1.shape
    _, H2, W2, _ = fmap2.shape
    S = coords.shape[1]
    g1 = torch.empty_like(fmap1)
    g2 = torch.empty_like(fmap2)
    gc = torch.empty(B, S, H1, W1, 2, dtype=torch.float32, device=fmap1.device)
    rc = _lib.load().vipe_altcorr_backward(fmap1.data_ptr(), fmap2.data_ptr(), coords.data_ptr(),
                                           corr_grad.data_ptr(), B, S, H1, W1, H2, W2, C, int(radius),
                                           int(bool(exact_coords_grad)), g1.data_ptr(), g2.data_ptr(), gc.data_ptr(),
                                           _lib.stream_of(fmap1))
    _lib.check(rc, "droid_net_ext.altcorr_backward")
    return [g1, g2, gc]


def altcorr_index_forward(fmap1, fmap2_pyramid, coords, ii, jj, radius):
    """fmap1 (B,Nf,H,W,C); fmap2_pyramid: list of (B,Nf,H_l,W_l,C); coords (B,M,H,W,2);
    ii, jj (M,) int64 -> [corr (B, M, L*(2r+1)^2, H, W) float32]."""
    _check("fmap1", fmap1)
    _check("coords", coords)
    _check("ii", ii)
    _check("jj", jj)
    _lib.require_dtype("coords", coords, torch.float32)
    _lib.require_dtype("ii", ii, torch.int64)
    _lib.require_dtype("jj", jj, torch.int64)
    levels = list(fmap2_pyramid)
    for l, f in enumerate(levels):
        _check(f"fmap2_pyramid[{l}]", f)
        if f.dtype != fmap1.dtype:
            raise RuntimeError("pyramid levels must share fmap1's dtype")
    B, Nf, H, W, C = fmap1.shape
    M = coords.shape[1]
    L = len(levels)
    rd = 2 * int(radius) + 1
    corr = torch.empty(B, M, L * rd * rd, H, W, dtype=torch.float32, device=fmap1.device)
    ptrs = (ctypes.c_void_p * L)(*[f.data_ptr() for f in levels])
    h2 = (ctypes.c_int * L)(*[f.shape[2] for f in levels])
    w2 = (ctypes.c_int * L)(*[f.shape[3] for f in levels])
    rc = _lib.load().vipe_altcorr_index_forward(_lib.DTYPE_CODE[fmap1.dtype], fmap1.data_ptr(), ptrs, h2, w2, L,
                                                coords.data_ptr(), ii.data_ptr(), jj.data_ptr(), B, Nf, M, H, W, C,
                                                int(radius), corr.data_ptr(), _lib.stream_of(fmap1))
    _lib.check(rc, "droid_net_ext.altcorr_index_forward")
    return [corr]


def altcorr_index_backward(fmap1, fmap2_pyramid, coords, ii, jj, corr_grad, radius, exact_coords_grad=False):
    """Adjoint of altcorr_index_forward (not in the reference) -> [fmap1_grad (B,Nf,H,W,C) f32,
    [level grads (B,Nf,H_l,W_l,C) f32], coords_grad (B,M,H,W,2) f32 (zeros unless exact_coords_grad)]."""
    for n, t in (("fmap1", fmap1), ("coords", coords), ("ii", ii), ("jj", jj), ("corr_grad", corr_grad)):
        _check(n, t)
    _lib.require_dtype("coords", coords, torch.float32)
    _lib.require_dtype("corr_grad", corr_grad, torch.float32)
    _lib.require_dtype("ii", ii, torch.int64)
    _lib.require_dtype("jj", jj, torch.int64)
    levels = list(fmap2_pyramid)
    for l, f in enumerate(levels):
        _check(f"fmap2_pyramid[{l}]", f)
        if f.dtype != fmap1.dtype:
            raise RuntimeError("pyramid levels must share fmap1's dtype")
    B, Nf, H, W, C = fmap1.shape
    M = coords.shape[1]
    L = len(levels)
    dev = fmap1.device
    g1 = torch.empty(B, Nf, H, W, C, dtype=torch.float32, device=dev)
    gl = [torch.empty(f.shape, dtype=torch.float32, device=dev) for f in levels]
    gc = torch.empty(B, M, H, W, 2, dtype=torch.float32, device=dev)
    ptrs = (ctypes.c_void_p * L)(*[f.data_ptr() for f in levels])
    gptrs = (ctypes.c_void_p * L)(*[g.data_ptr() for g in gl])
    h2 = (ctypes.c_int * L)(*[f.shape[2] for f in levels])
    w2 = (ctypes.c_int * L)(*[f.shape[3] for f in levels])
    rc = _lib.load().vipe_altcorr_index_backward(_lib.DTYPE_CODE[fmap1.dtype], fmap1.data_ptr(), ptrs, h2, w2, L,
                                                 coords.data_ptr(), ii.data_ptr(), jj.data_ptr(),
                                                 corr_grad.data_ptr(), B, Nf, M, H, W, C, int(radius),
                                                 int(bool(exact_coords_grad)), g1.data_ptr(), gptrs, gc.data_ptr(),
                                                 _lib.stream_of(fmap1))
    _lib.check(rc, "droid_net_ext.altcorr_index_backward")
    return [g1, gl, gc]
