"""The tcgen05 adjoint of the correlation-volume pyramid (vipe_corr_volume_backward).

d fmap1 = (1/16) fmap2 Gt^T, d fmap2 = (1/16) fmap1 Gt with Gt the unpooled sum of the
level gradients, against
  * the FP64 oracle (oracle/corr.py corr_pyramid_backward: every level gradient spread back
    to level 0, then both products), on the operands the forward multiplied;
  * torch autograd of the reference's eager construction (droid_net.py:56-69, 94-102:
    matmul of the /4 maps, then avg_pool2d per level) in FP64 on the GPU.
Tolerances, relative to the largest gradient entry: FP32 level gradients (split TF32
products) 2e-5; FP16 gradients (Gt rounded to FP16 once) 2e-3; BF16 1.5e-2.
"""

import numpy as np
import pytest
import torch
import torch.nn.functional as F

import oracle.corr as oc

pytestmark = pytest.mark.gpu


def _backward(f1, f2, grads, map_dtype):
    """(d fmap1, d fmap2) as the entry point writes them: FP32, before any cast to the map dtype."""
    import ctypes

    from vipe_b200 import _lib

    num, C, H, W = f1.shape
    g1 = torch.empty(num, C, H, W, device="cuda")
    g2 = torch.empty(num, C, H, W, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    ptrs = (ctypes.c_void_p * len(grads))(*[g.data_ptr() for g in grads])
    rc = _lib.load().vipe_corr_volume_backward(
        _lib.DTYPE_CODE[map_dtype], _lib.DTYPE_CODE[grads[0].dtype], f1.contiguous().data_ptr(),
        f2.contiguous().data_ptr(), ptrs, num, C, H, W, len(grads), g1.data_ptr(), g2.data_ptr(), st.data_ptr(),
        torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, "vipe_corr_volume_backward")
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return g1, g2


@pytest.mark.parametrize("map_dtype,grad_dtype,tol", [(torch.float16, torch.float16, 2e-3),
                                                      (torch.bfloat16, torch.bfloat16, 1.5e-2),
                                                      (torch.bfloat16, torch.float32, 2e-5),
                                                      (torch.float16, torch.float32, 2e-5)])
@pytest.mark.parametrize("shape,L", [((3, 128, 48, 64), 4), ((2, 96, 16, 32), 3), ((2, 64, 8, 16), 1)])
def test_volume_backward_vs_fp64_oracle(map_dtype, grad_dtype, tol, shape, L):
    g = torch.Generator().manual_seed(50)
    num, C, H, W = shape
    f1 = (torch.randn(num, C, H, W, generator=g) / C**0.5).to(map_dtype)
    f2 = (torch.randn(num, C, H, W, generator=g) / C**0.5).to(map_dtype)
    grads = [torch.randn(num, H * W, H >> l, W >> l, generator=g).to(grad_dtype) for l in range(L)]
    d1, d2 = _backward(f1.cuda(), f2.cuda(), [x.cuda() for x in grads], map_dtype)
    w1, w2 = oc.corr_pyramid_backward(f1.double().numpy(), f2.double().numpy(),
                                      [x.double().numpy() for x in grads])
    for got, want in ((d1, w1), (d2, w2)):
        got = got.double().cpu().numpy()
        assert np.abs(got - want).max() <= tol * np.abs(want).max()


def test_volume_backward_vs_autograd_of_the_reference_ops():
    """Config 2's shapes on a 4-edge slice (128 channels, 48x64, 4 levels), FP32 level gradients."""
    g = torch.Generator(device="cuda").manual_seed(51)
    num, C, H, W = 4, 128, 48, 64
    f1 = (torch.randn(num, C, H, W, generator=g, device="cuda") / C**0.5).bfloat16()
    f2 = (torch.randn(num, C, H, W, generator=g, device="cuda") / C**0.5).bfloat16()
    grads = [torch.randn(num, H * W, H >> l, W >> l, generator=g, device="cuda") for l in range(4)]
    d1, d2 = _backward(f1, f2, grads, torch.bfloat16)
    a = f1.double().requires_grad_()
    b = f2.double().requires_grad_()
    v = torch.matmul((a / 4).view(num, C, H * W).transpose(1, 2), (b / 4).view(num, C, H * W))
    v = v.view(num * H * W, 1, H, W)
    loss = 0
    for l in range(4):
        loss = loss + (v.view(num, H * W, H >> l, W >> l) * grads[l].double()).sum()
        v = F.avg_pool2d(v, 2, stride=2)
    loss.backward()
    for got, want in ((d1, a.grad), (d2, b.grad)):
        assert (got.double() - want).abs().max() <= 2e-5 * want.abs().max()


def _set_generic(on):
    from vipe_b200 import _lib

    _lib.load().vipe_corr_volume_backward_force_generic(int(on))


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
@pytest.mark.parametrize("shape,L", [((3, 128, 48, 64), 4), ((2, 96, 16, 64), 3), ((1, 128, 8, 128), 4),
                                     ((2, 64, 8, 64), 1), ((2, 128, 16, 64), 2)])
def test_tma_kernel_matches_producer_kernel(dtype, shape, L):
    """The TMA-fed kernel (16-bit maps and gradients of one type, W % 64 == 0) against the
    producer-formed kernel on the same inputs: both round Gt = G_0 + sum_l G_l / 4^l once, in
    the same order, and accumulate the same K blocks in the same order, so the FP32 gradients
    agree to the bit."""
    g = torch.Generator(device="cuda").manual_seed(52)
    num, C, H, W = shape
    f1 = (torch.randn(num, C, H, W, generator=g, device="cuda") / C**0.5).to(dtype)
    f2 = (torch.randn(num, C, H, W, generator=g, device="cuda") / C**0.5).to(dtype)
    grads = [torch.randn(num, H * W, H >> l, W >> l, generator=g, device="cuda").to(dtype) for l in range(L)]
    fast = _backward(f1, f2, grads, dtype)
    _set_generic(True)
    try:
        slow = _backward(f1, f2, grads, dtype)
    finally:
        _set_generic(False)
    for a, b in zip(fast, slow):
        torch.testing.assert_close(a, b, atol=0, rtol=0)


@pytest.mark.parametrize("shape,L", [((2, 96, 16, 64), 3), ((1, 128, 8, 128), 4)])
def test_tma_kernel_vs_fp64_oracle(shape, L):
    g = torch.Generator().manual_seed(53)
    num, C, H, W = shape
    f1 = (torch.randn(num, C, H, W, generator=g) / C**0.5).half()
    f2 = (torch.randn(num, C, H, W, generator=g) / C**0.5).half()
    grads = [torch.randn(num, H * W, H >> l, W >> l, generator=g).half() for l in range(L)]
    d1, d2 = _backward(f1.cuda(), f2.cuda(), [x.cuda() for x in grads], torch.float16)
    w1, w2 = oc.corr_pyramid_backward(f1.double().numpy(), f2.double().numpy(), [x.double().numpy() for x in grads])
    for got, want in ((d1, w1), (d2, w2)):
        got = got.double().cpu().numpy()
        assert np.abs(got - want).max() <= 2e-3 * np.abs(want).max()
