"""corr_ext — drop-in for the reference's ``vipe.ext.corr_ext`` pybind module.

Reference bindings: vipe csrc/corr_ext/correlation_sampler.cpp:82-85 (``forward``,
``backward``), used through vipe/ext/corr/spatial_correlation_sampler.py by the AOT
tracker's attention layers.  Same names, positional arguments and returns:

    forward(input1, input2, kH, kW, patchH, patchW, padH, padW, dilationH, dilationW,
            dilation_patchH, dilation_patchW, dH, dW) -> output (N, patchH, patchW, oH, oW)
    backward(input1, input2, grad_output, <the same 12 ints>) -> [grad_input1, grad_input2]

CUDA tensors only (the reference also has a CPU loop; this library has no CPU path).
Accumulation is FP32 (FP64 for double maps); the reference's GPU kernel accumulates in
the map type.
"""

from __future__ import annotations

import torch

from .. import _lib

_DT = (torch.float32, torch.float64, torch.float16, torch.bfloat16)


def _prep(name, t):
    _lib.require_cuda(name, t)
    _lib.require_contiguous(name, t)
    _lib.require_dtype(name, t, *_DT)


def _out_size(H, W, kH, kW, padH, padW, dilationH, dilationW, dH, dW):
    oH = (H + 2 * padH - ((kH - 1) * dilationH + 1)) // dH + 1
    oW = (W + 2 * padW - ((kW - 1) * dilationW + 1)) // dW + 1
    return oH, oW


def forward(input1, input2, kH, kW, patchH, patchW, padH, padW, dilationH, dilationW, dilation_patchH,
            dilation_patchW, dH, dW):
    _prep("input1", input1)
    _prep("input2", input2)
    if input1.shape != input2.shape or input1.dtype != input2.dtype:
        raise RuntimeError("input1 and input2 must have the same shape and dtype")
    N, C, H, W = input1.shape
    oH, oW = _out_size(H, W, kH, kW, padH, padW, dilationH, dilationW, dH, dW)
    out = torch.empty(N, patchH, patchW, oH, oW, dtype=input1.dtype, device=input1.device)
    rc = _lib.load().vipe_corr_sample_forward(
        _lib.DTYPE_CODE[input1.dtype], input1.data_ptr(), input2.data_ptr(), N, C, H, W, kH, kW, patchH, patchW, padH,
        padW, dilationH, dilationW, dilation_patchH, dilation_patchW, dH, dW, out.data_ptr(), _lib.stream_of(input1))
    _lib.check(rc, "corr_ext.forward")
    return out


def backward(input1, input2, grad_output, kH, kW, patchH, patchW, padH, padW, dilationH, dilationW, dilation_patchH,
             dilation_patchW, dH, dW):
    _prep("input1", input1)
    _prep("input2", input2)
    _prep("grad_output", grad_output)
    N, C, H, W = input1.shape
    g1 = torch.empty_like(input1)
    g2 = torch.empty_like(input2)
    rc = _lib.load().vipe_corr_sample_backward(
        _lib.DTYPE_CODE[input1.dtype], input1.data_ptr(), input2.data_ptr(), grad_output.data_ptr(), N, C, H, W, kH,
        kW, patchH, patchW, padH, padW, dilationH, dilationW, dilation_patchH, dilation_patchW, dH, dW,
        g1.data_ptr(), g2.data_ptr(), _lib.stream_of(input1))
    _lib.check(rc, "corr_ext.backward")
    return [g1, g2]
