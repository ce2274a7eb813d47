"""AltCorrBlock's channels-last feature pyramid kernel against the reference's eager construction.

The reference (vipe/slam/networks/droid_net.py:130-142) builds the pyramid with torch:
fmaps / 4.0, then per level permute(0, 2, 3, 1).contiguous() and avg_pool2d(2, stride 2).
vipe_corr_pyramid_nhwc must give the same levels bit for bit (it rounds every level to the
element type before pooling the next, summing each window in FP32 in avg_pool2d's order),
for FP16, BF16 and FP32 maps, odd sizes (floor pooling) included.  The adjoint is held to
torch autograd of that eager construction.
"""

import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def _eager_levels(fmaps, L):
    f = fmaps / 4.0
    out = []
    for _ in range(L):
        out.append(f.permute(0, 2, 3, 1).contiguous())
        f = F.avg_pool2d(f, 2, stride=2)
    return out


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16, torch.float32])
@pytest.mark.parametrize("shape,L", [((6, 128, 48, 64), 4), ((3, 64, 47, 61), 4), ((2, 8, 20, 36), 3),
                                     ((1, 256, 9, 17), 2)])
def test_pyramid_bit_exact_vs_eager_reference(dtype, shape, L):
    from vipe_b200.droid_corr import _pyramid_levels

    g = torch.Generator(device="cuda").manual_seed(31)
    fm = (torch.randn(shape, generator=g, device="cuda") * 3).to(dtype)
    got = _pyramid_levels(fm, L)
    want = _eager_levels(fm, L)
    assert len(got) == L
    for a, b in zip(got, want):
        assert a.shape == b.shape and a.dtype == b.dtype
        torch.testing.assert_close(a, b, atol=0, rtol=0)


@pytest.mark.parametrize("dtype,tol", [(torch.float32, 1e-6), (torch.float16, 2e-3), (torch.bfloat16, 1e-2)])
def test_pyramid_backward_vs_autograd(dtype, tol):
    from vipe_b200.droid_corr import FeaturePyramid

    g = torch.Generator(device="cuda").manual_seed(32)
    B, N, C, H, W = 1, 3, 128, 47, 62
    base = torch.randn(B * N, C, H, W, generator=g, device="cuda").to(dtype)
    R = [torch.randn(B * N, H >> l, W >> l, C, generator=g, device="cuda") for l in range(4)]
    x = base.clone().requires_grad_()
    lv = FeaturePyramid.apply(x, 4)
    sum((a.float() * r).sum() for a, r in zip(lv, R)).backward()
    y = base.double().clone().requires_grad_()  # FP64 autograd of the reference's eager ops
    sum((a * r.double()).sum() for a, r in zip(_eager_levels(y, 4), R)).backward()
    assert x.grad.dtype == dtype
    scale = y.grad.abs().max()
    assert (x.grad.double() - y.grad).abs().max() <= tol * scale


def test_altcorrblock_uses_the_kernel_pyramid():
    from vipe_b200.droid_corr import AltCorrBlock

    g = torch.Generator(device="cuda").manual_seed(33)
    fm = torch.randn(1, 4, 128, 48, 64, generator=g, device="cuda").half()
    blk = AltCorrBlock(fm)
    for a, b in zip(blk.pyramid, _eager_levels(fm.view(4, 128, 48, 64), 4)):
        torch.testing.assert_close(a.view(b.shape), b, atol=0, rtol=0)
