"""Python front of the tcgen05 correlation-volume build (vipe_corr_volume_build).

corr_volume_pyramid(fmap1, fmap2, num_levels) returns the CorrBlock pyramid:
level l = avg_pool2d^l((fmap1/4)^T (fmap2/4)) over the target axes, shaped
(num, H*W, H >> l, W >> l).  fmap1, fmap2: (num, C, H, W) CUDA tensors (float16
stays FP16 on the tensor cores; bfloat16 and float32 run as BF16), C <= 128,
H % 8 == 0 and W % 8 == 0 (the pooled pyramid closes inside 8 x 8 target
blocks).
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib


def corr_volume_pyramid(fmap1, fmap2, num_levels=4, out_dtype=torch.float32, compute_dtype=None, check=True):
    for name, t in (("fmap1", fmap1), ("fmap2", fmap2)):
        _lib.require_cuda(name, t)
    if fmap1.shape != fmap2.shape or fmap1.dim() != 4:
        raise RuntimeError("fmap1 and fmap2 must both be (num, C, H, W)")
    if compute_dtype is not None:
        fmap1 = fmap1.to(compute_dtype)
        fmap2 = fmap2.to(compute_dtype)
    fmap1 = fmap1.contiguous()
    fmap2 = fmap2.contiguous()
    if fmap2.dtype != fmap1.dtype:
        fmap2 = fmap2.to(fmap1.dtype)
    num, C, H, W = fmap1.shape
    if out_dtype not in (torch.float32, torch.float16, torch.bfloat16):
        raise RuntimeError(f"unsupported volume dtype {out_dtype}")
    dev = fmap1.device
    lib = _lib.load()
    ws_bytes = lib.vipe_corr_volume_workspace_size(num, C, H, W)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    levels = [torch.empty(num, H * W, H >> l, W >> l, dtype=out_dtype, device=dev) for l in range(num_levels)]
    ptrs = (ctypes.c_void_p * num_levels)(*[t.data_ptr() for t in levels])
    rc = lib.vipe_corr_volume_build(_lib.DTYPE_CODE[fmap1.dtype], _lib.DTYPE_CODE[out_dtype], fmap1.data_ptr(),
                                    fmap2.data_ptr(), num, C, H, W, num_levels, ptrs, ws.data_ptr(), ws_bytes,
                                    _lib.stream_of(fmap1))
    _lib.check(rc, "corr_volume_build")
    if check and int(ws[:4].view(torch.int32).item()) != 0:
        raise RuntimeError("corr_volume_build: a bounded wait expired on the device; the volume is incomplete")
    return levels


