"""The CorrBlock lookup fused with the update operator's first correlation layer.

vipe_corr_encoder_lookup computes ReLU(conv1x1(lookup)) — UpdateModule.corr_encoder[0:2]
(vipe/slam/networks/droid_net.py:455-460) applied to CorrBlock's 196-channel radius-3 lookup
(:94-102) — in one tcgen05 kernel.  Held to:
  * the unfused composition on the same GPU: vipe_b200's own lookup (corr_index_forward per
    level, FP16/BF16 output) followed by an FP32 1x1 convolution and ReLU, rounded to the
    volume type: within 2 ulps of the output type relative to the largest output;
  * the reference's path: the reference's own corr_index_forward (compiled from its sources,
    oracle/_ref) per level, then torch's conv2d in the volume type, ReLU: within 1e-2 of the
    largest output (the reference rounds the lookup after every tap).
"""

import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def _setup(dtype, N, H, W, seed, spill=0.0):
    from vipe_b200.droid_corr import CorrBlock

    g = torch.Generator(device="cuda").manual_seed(seed)
    f1 = (torch.randn(1, N, 128, H, W, generator=g, device="cuda") / 4).to(dtype)
    f2 = (torch.randn(1, N, 128, H, W, generator=g, device="cuda") / 4).to(dtype)
    blk = CorrBlock(f1, f2, num_levels=4, radius=3, out_dtype=dtype)
    yy, xx = torch.meshgrid(torch.arange(H, device="cuda"), torch.arange(W, device="cuda"), indexing="ij")
    coords = torch.stack([xx, yy], -1).float()[None, None].repeat(1, N, 1, 1, 1)
    coords = coords + 1.5 * torch.randn(coords.shape, generator=g, device="cuda")
    if spill:
        coords[:, :, :3] -= spill  # windows partly or wholly off the map
    w = (torch.randn(128, 196, 1, 1, generator=g, device="cuda") / 14.0)
    b = 0.1 * torch.randn(128, generator=g, device="cuda")
    return blk, coords, w, b


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
@pytest.mark.parametrize("N,H,W,spill", [(6, 48, 64, 0.0), (3, 16, 32, 9.0), (2, 24, 40, 3.0)])
def test_fused_matches_unfused_composition(dtype, N, H, W, spill):
    from vipe_b200.droid_corr import corr_encoder_input

    blk, coords, w, b = _setup(dtype, N, H, W, seed=60 + H, spill=spill)
    got = corr_encoder_input(blk, coords, w, b)
    corr = blk(coords).view(N, 196, H, W)  # vipe_b200's lookup, rounded to the volume type
    want = F.relu(F.conv2d(corr.float(), w.to(dtype).float(), b)).to(dtype)
    assert got.shape == want.shape and got.dtype == dtype
    ulp = 2.0 ** (-10 if dtype == torch.float16 else -7)
    assert (got.float() - want.float()).abs().max() <= 2 * ulp * want.float().abs().max()


@pytest.mark.parametrize("bias", [True, False])
def test_fused_matches_reference_path(bias):
    from oracle import build_ref
    from vipe_b200.droid_corr import corr_encoder_input

    ref = build_ref.load("ref_droid_net_ext")
    N, H, W = 4, 48, 64
    blk, coords, w, b = _setup(torch.float16, N, H, W, seed=70)
    b = b if bias else None
    got = corr_encoder_input(blk, coords, w, b)
    c = coords[0].permute(0, 3, 1, 2).contiguous()
    corr = torch.cat([ref.corr_index_forward(lv.contiguous(), (c / 2**l).contiguous(), 3)[0].view(N, 49, H, W)
                      for l, lv in enumerate(blk.corr_pyramid)], 1)
    want = F.relu(F.conv2d(corr, w.half(), None if b is None else b.half()))
    assert (got.float() - want.float()).abs().max() <= 1e-2 * want.float().abs().max()
