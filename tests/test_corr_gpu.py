"""Correlation ops on the GPU against the FP64 oracle (oracle/corr.py).

* lookups (corr_index fwd/bwd, altcorr fwd/bwd, altcorr_index fwd) in f32
  (atol 1e-4), f16 inputs (atol 2e-3 on O(1) outputs), f64 (atol 1e-10);
  out-of-map coordinates exercise the zero padding;
* the reference's own check (tests/test_altcorr_indexed.py): 7 fp16 frames,
  128 channels, 48x64, 5 edges, coords = grid + 0.4 N(0,1), seed 2028 —
  indexed vs per-level lookup at atol 2e-4, rtol 1e-4;
* the tcgen05 volume build + fused pyramid vs the FP64 oracle evaluated on the
  same BF16 / FP16-rounded inputs: |err| <= 1e-4 * max|V| (FP32 accumulation).
"""

import numpy as np
import pytest
import torch

import oracle.corr as oc

pytestmark = pytest.mark.gpu


def _dne():
    from vipe_b200.ext import droid_net_ext

    return droid_net_ext


def _grid_coords(B, H, W, gen, sigma, spill=0.0):
    yy, xx = torch.meshgrid(torch.arange(H), torch.arange(W), indexing="ij")
    c = torch.stack([xx, yy], 0).float()[None].repeat(B, 1, 1, 1)
    c = c + sigma * torch.randn(c.shape, generator=gen)
    if spill:
        c[:, :, :2] -= spill  # push some lookups off the map
    return c


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16, torch.float64])
def test_corr_index_forward_backward(dtype):
    g = torch.Generator().manual_seed(11)
    B, h1, w1, h2, w2 = 2, 6, 8, 6, 8
    vol = torch.randn(B, h1, w1, h2, w2, generator=g)
    coords = _grid_coords(B, h1, w1, g, 1.5, spill=5.0)
    out = _dne().corr_index_forward(vol.to(dtype).cuda(), coords.cuda(), 3)[0]
    want = oc.corr_index_forward(vol.to(dtype).double().numpy(), coords.numpy(), 3)
    tol = {torch.float32: 1e-5, torch.float16: 4e-3, torch.float64: 1e-12}[dtype]
    np.testing.assert_allclose(out.double().cpu().numpy(), want, atol=tol)
    grad = torch.randn(B, 7, 7, h1, w1, generator=g)
    vg = _dne().corr_index_backward(vol.to(dtype).cuda(), coords.cuda(), grad.to(dtype).cuda(), 3)[0]
    wv = oc.corr_index_backward(vol.shape, coords.numpy(), grad.to(dtype).double().numpy(), 3)
    np.testing.assert_allclose(vg.double().cpu().numpy(), wv, atol=tol * 4)


@pytest.mark.parametrize("dtype,w2", [(torch.float16, 32), (torch.bfloat16, 16), (torch.float32, 12),
                                      (torch.float32, 6), (torch.float16, 6)])
def test_corr_index_forward_vector_and_scalar_paths(dtype, w2):
    """Radius 3 takes the 16-byte row-chunk path when w2 * size is a multiple of 16 (w2 = 32, 16, 12
    here) and the element path otherwise (w2 = 6); windows straddle every border, and far-away
    coordinates read only zeros."""
    g = torch.Generator().manual_seed(20)
    B, h1, w1, h2 = 2, 5, 7, 9
    vol = torch.randn(B, h1, w1, h2, w2, generator=g)
    coords = torch.stack([torch.rand(B, h1, w1, generator=g) * (w2 + 10) - 5,
                          torch.rand(B, h1, w1, generator=g) * (h2 + 10) - 5], 1)
    coords[0, :, 0, 0] = 1e9  # far outside: all taps zero
    coords[1, :, 1, 1] = -3e9
    out = _dne().corr_index_forward(vol.to(dtype).cuda(), coords.cuda(), 3)[0]
    want = oc.corr_index_forward(vol.to(dtype).double().numpy(), coords.double().numpy(), 3)
    tol = {torch.float32: 1e-5, torch.float16: 4e-3, torch.bfloat16: 3e-2}[dtype]
    np.testing.assert_allclose(out.double().cpu().numpy(), want, atol=tol)
    assert float(out[0, :, :, 0, 0].abs().max()) == 0.0 and float(out[1, :, :, 1, 1].abs().max()) == 0.0


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
def test_altcorr_forward(dtype):
    g = torch.Generator().manual_seed(12)
    B, S, H, W, C = 2, 2, 8, 16, 64
    f1 = torch.randn(B, H, W, C, generator=g) / 8
    f2 = torch.randn(B, H, W, C, generator=g) / 8
    coords = torch.stack([_grid_coords(B, H, W, g, 1.5, spill=4.0).permute(0, 2, 3, 1) for _ in range(S)], 1)
    out = _dne().altcorr_forward(f1.to(dtype).cuda(), f2.to(dtype).cuda(), coords.contiguous().cuda(), 3)[0]
    want = oc.altcorr_forward(f1.to(dtype).double().numpy(), f2.to(dtype).double().numpy(), coords.numpy(), 3)
    tol = 1e-5 if dtype == torch.float32 else 3e-3
    np.testing.assert_allclose(out.double().cpu().numpy(), want, atol=tol)


@pytest.mark.parametrize("exact", [False, True])
def test_altcorr_backward(exact):
    g = torch.Generator().manual_seed(13)
    B, S, H, W, C = 1, 2, 6, 8, 32
    f1 = torch.randn(B, H, W, C, generator=g) / 4
    f2 = torch.randn(B, H, W, C, generator=g) / 4
    coords = torch.stack([_grid_coords(B, H, W, g, 1.2).permute(0, 2, 3, 1) for _ in range(S)], 1).contiguous()
    grad = torch.randn(B, S, 49, H, W, generator=g)
    g1, g2, gc = _dne().altcorr_backward(f1.cuda(), f2.cuda(), coords.cuda(), grad.cuda(), 3, exact)
    w1, w2, wc = oc.altcorr_backward(f1.numpy(), f2.numpy(), coords.numpy(), grad.numpy(), 3, exact_coords=exact)
    np.testing.assert_allclose(g1.cpu().numpy(), w1, atol=1e-4)
    np.testing.assert_allclose(g2.cpu().numpy(), w2, atol=1e-4)
    np.testing.assert_allclose(gc.cpu().numpy(), wc, atol=1e-4)
    if not exact:
        assert float(gc.abs().max()) == 0.0  # reference returns zeros (altcorr_kernel.cu:440)


def test_altcorr_index_matches_oracle_and_reference_property():
    # reference tests/test_altcorr_indexed.py:23-48
    from vipe_b200.droid_corr import AltCorrBlock

    torch.manual_seed(2028)
    batch, n_frames, channels, height, width, n_edges = 1, 7, 128, 48, 64, 5
    fmaps = torch.randn(batch, n_frames, channels, height, width, device="cuda", dtype=torch.float16)
    yy, xx = torch.meshgrid(torch.arange(height, device="cuda"), torch.arange(width, device="cuda"), indexing="ij")
    coords = torch.stack([xx, yy], dim=-1).float()[None].repeat(batch, n_edges, 1, 1, 1)
    coords = coords + 0.4 * torch.randn_like(coords)
    ii = torch.tensor([0, 1, 2, 3, 4], device="cuda", dtype=torch.long)
    jj = torch.tensor([1, 2, 3, 4, 5], device="cuda", dtype=torch.long)
    corr = AltCorrBlock(fmaps)
    cs = coords.unsqueeze(dim=-2)
    reference = corr.corr_fn_reference(cs, ii, jj)
    indexed = corr.corr_fn_indexed(cs, ii, jj)
    torch.testing.assert_close(indexed, reference, atol=2e-4, rtol=1e-4)
    default = corr(coords, ii, jj)
    torch.testing.assert_close(default, reference.squeeze(dim=-1), atol=2e-4, rtol=1e-4)
    # against the FP64 oracle on the same fp16 pyramid (edges 0..1 to keep the CPU side quick)
    levels = [p.double().cpu().numpy() for p in corr.pyramid]
    want = oc.altcorr_index_forward(levels[0], levels, coords[:, :2].cpu().numpy(), [0, 1], [1, 2], 3)
    np.testing.assert_allclose(indexed[:, :2, ..., 0].double().cpu().numpy(), want, atol=5e-4)


@pytest.mark.parametrize(
    "in_dtype,out_dtype,shape",
    [
        (torch.bfloat16, torch.float32, (3, 128, 16, 32)),
        (torch.float16, torch.float32, (3, 128, 16, 32)),
        (torch.bfloat16, torch.float16, (2, 128, 16, 64)),
        (torch.float16, torch.bfloat16, (2, 64, 8, 16)),
        (torch.float32, torch.float32, (2, 96, 8, 8)),
        (torch.bfloat16, torch.float32, (2, 128, 8, 24)),
        # 16-bit output, 32-wide target blocks: level 0 leaves the epilogue as 32-byte row stores
        (torch.bfloat16, torch.float16, (2, 128, 48, 64)),
        (torch.float16, torch.bfloat16, (1, 128, 16, 64)),
        # 64-wide 16-bit: one 64-channel box (A read from fmap1 directly), and C = 96 (padded to 128:
        # both operands packed, full-row TMA-store epilogue)
        (torch.bfloat16, torch.bfloat16, (2, 64, 16, 64)),
        (torch.float16, torch.float16, (1, 96, 16, 64)),
    ],
)
def test_volume_build_pyramid(in_dtype, out_dtype, shape):
    from vipe_b200.corr_build import corr_volume_pyramid

    g = torch.Generator().manual_seed(14)
    num, C, H, W = shape
    f1 = torch.randn(num, C, H, W, generator=g) / np.sqrt(C) * 4
    f2 = torch.randn(num, C, H, W, generator=g) / np.sqrt(C) * 4
    op = torch.bfloat16 if in_dtype == torch.float32 else in_dtype  # float32 inputs run as BF16 operands
    levels = corr_volume_pyramid(f1.to(in_dtype).cuda(), f2.to(in_dtype).cuda(), 4, out_dtype=out_dtype)
    want = oc.corr_pyramid(f1.to(op).double().numpy(), f2.to(op).double().numpy(), 4)
    # FP32 accumulation of pre-rounded operands; the stored volume adds its own rounding
    tol = {torch.float32: 1e-4, torch.float16: 2e-3, torch.bfloat16: 1e-2}[out_dtype]
    for l, (got, w) in enumerate(zip(levels, want)):
        got = got.cpu().double().numpy().reshape(w.shape)
        scale = np.abs(w).max()
        err = np.abs(got - w).max()
        assert err <= tol * scale, (l, err, scale)


def test_volume_build_shapes_and_corrblock():
    from vipe_b200.droid_corr import CorrBlock

    g = torch.Generator().manual_seed(15)
    B, N, C, H, W = 1, 2, 128, 8, 16
    f1 = (torch.randn(B, N, C, H, W, generator=g) / 4).half().cuda()
    f2 = (torch.randn(B, N, C, H, W, generator=g) / 4).half().cuda()
    cb = CorrBlock(f1, f2, num_levels=4, radius=3)
    assert [tuple(p.shape) for p in cb.corr_pyramid] == [(2, 8, 16, 8, 16), (2, 8, 16, 4, 8), (2, 8, 16, 2, 4),
                                                          (2, 8, 16, 1, 2)]
    coords = _grid_coords(B * N, H, W, g, 1.0).permute(0, 2, 3, 1).reshape(B, N, H, W, 2).cuda()
    out = cb(coords)
    assert out.shape == (B, N, 4 * 49, H, W)
    pyr = oc.corr_pyramid(f1[0].double().cpu().numpy(), f2[0].double().cpu().numpy(), 4)
    c4 = coords[0].permute(0, 3, 1, 2).cpu().numpy()
    want = np.concatenate([oc.corr_index_forward(pyr[l], c4 / 2**l, 3).reshape(N, 49, H, W) for l in range(4)], 1)
    np.testing.assert_allclose(out[0].double().cpu().numpy(), want, atol=1e-2)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16, torch.float64])
def test_corr_index_coords_backward(dtype):
    g = torch.Generator().manual_seed(16)
    B, h1, w1, h2, w2 = 2, 6, 8, 6, 8
    vol = torch.randn(B, h1, w1, h2, w2, generator=g)
    coords = _grid_coords(B, h1, w1, g, 1.5, spill=5.0)
    grad = torch.randn(B, 7, 7, h1, w1, generator=g)
    out = _dne().corr_index_coords_backward(vol.to(dtype).cuda(), coords.cuda(), grad.to(dtype).cuda(), 3)[0]
    want = oc.corr_index_coords_backward(vol.to(dtype).double().numpy(), coords.numpy(),
                                         grad.to(dtype).double().numpy(), 3)
    tol = {torch.float32: 1e-4, torch.float16: 2e-2, torch.float64: 1e-5}[dtype]  # f64 result is stored as f32
    np.testing.assert_allclose(out.double().cpu().numpy(), want, atol=tol, rtol=1e-5)


@pytest.mark.parametrize("dtype,W", [(torch.float32, 32), (torch.float16, 32), (torch.float16, 64)])
def test_corrblock_gradients_fmaps_and_coords(dtype, W):
    """CorrBlock forward + backward: gradients to both feature maps and to the coordinates
    against the FP64 oracle (lookup adjoint per level, then the pyramid backward) on the
    operands the tensor cores multiplied."""
    from vipe_b200.droid_corr import CorrBlock, CorrSampler

    g = torch.Generator().manual_seed(17)
    B, N, C, H = 1, 2, 64, 16  # W = 64 with 16-bit maps: full-row tiles, A operand read from fmap1
    f1 = (torch.randn(B, N, C, H, W, generator=g) / 2).to(dtype).cuda().requires_grad_()
    f2 = (torch.randn(B, N, C, H, W, generator=g) / 2).to(dtype).cuda().requires_grad_()
    coords = _grid_coords(B * N, H, W, g, 1.5).permute(0, 2, 3, 1).reshape(B, N, H, W, 2)
    coords = coords.cuda().requires_grad_()
    R = torch.randn(B, N, 4 * 49, H, W, generator=g)
    CorrSampler.exact_coords_grad = True
    try:
        # 16-bit inputs keep a 16-bit volume: lookup and level gradients in FP16, products in FP16
        out_dtype = torch.float32 if dtype == torch.float32 else dtype
        out = CorrBlock(f1, f2, num_levels=4, radius=3, out_dtype=out_dtype)(coords)
        (out * R.to(out_dtype).cuda()).sum().backward()
    finally:
        CorrSampler.exact_coords_grad = False
    op = torch.bfloat16 if dtype == torch.float32 else dtype
    a1 = f1.detach().to(op).double().cpu().numpy()[0]
    a2 = f2.detach().to(op).double().cpu().numpy()[0]
    pyr = oc.corr_pyramid(a1, a2, 4)
    c4 = coords.detach()[0].permute(0, 3, 1, 2).cpu().double().numpy()
    Rn = R[0].to(dtype).double().numpy().reshape(N, 4, 7, 7, H, W)
    lg, gc = [], np.zeros_like(c4)
    for l in range(4):
        lg.append(oc.corr_index_backward(pyr[l].shape, c4 / 2**l, Rn[:, l], 3))
        gc += oc.corr_index_coords_backward(pyr[l], c4 / 2**l, Rn[:, l], 3) / 2**l
    w1, w2 = oc.corr_pyramid_backward(a1, a2, lg)
    got1 = f1.grad[0].double().cpu().numpy()
    got2 = f2.grad[0].double().cpu().numpy()
    gotc = coords.grad[0].permute(0, 3, 1, 2).double().cpu().numpy()
    # FP32: FP32 products of FP32 level gradients; FP16: every level gradient and product rounded to FP16
    tol = 1e-4 if dtype == torch.float32 else 1e-2
    for got, want in ((got1, w1), (got2, w2)):
        assert np.abs(got - want).max() <= tol * np.abs(want).max()
    # the coordinate gradient differences neighbouring volume taps (FP32-accumulated on the GPU, FP16-stored
    # for FP16 inputs)
    ctol = 2e-3 if dtype == torch.float32 else 2e-2
    assert np.abs(gotc - gc).max() <= ctol * np.abs(gc).max()


@pytest.mark.parametrize("dtype,C", [(torch.float32, 32), (torch.float32, 30), (torch.float16, 64),
                                     (torch.bfloat16, 128)])
def test_altcorr_index_backward(dtype, C):
    g = torch.Generator().manual_seed(18)
    B, Nf, H, W, M = 1, 4, 16, 24, 5
    f = (torch.randn(B, Nf, H, W, C, generator=g) / 4).to(dtype)
    levels = [f]
    for _ in range(3):
        t = levels[-1].float().permute(0, 1, 4, 2, 3).reshape(B * Nf, C, levels[-1].shape[2], levels[-1].shape[3])
        t = torch.nn.functional.avg_pool2d(t, 2, stride=2)
        levels.append(t.reshape(B, Nf, C, t.shape[-2], t.shape[-1]).permute(0, 1, 3, 4, 2).contiguous().to(dtype))
    ii = torch.tensor([0, 1, 2, 0, 3])
    jj = torch.tensor([1, 2, 3, 2, 2])  # frames 0 and 2 are each used by two edges: overlapping scatters
    coords = _grid_coords(B * M, H, W, g, 1.5, spill=3.0).reshape(B, M, 2, H, W).permute(0, 1, 3, 4, 2).contiguous()
    grad = torch.randn(B, M, 4 * 49, H, W, generator=g)
    g1, gl, gc = _dne().altcorr_index_backward(f.cuda(), [lv.cuda() for lv in levels], coords.cuda(), ii.cuda(),
                                               jj.cuda(), grad.cuda(), 3, True)
    w1, wl, wc = oc.altcorr_index_backward(f.double().numpy(), [lv.double().numpy() for lv in levels],
                                           coords.numpy(), ii.numpy(), jj.numpy(), grad.numpy(), 3,
                                           exact_coords=True)
    np.testing.assert_allclose(g1.cpu().numpy(), w1, atol=2e-4)
    for a, b in zip(gl, wl):
        np.testing.assert_allclose(a.cpu().numpy(), b, atol=2e-4)
    np.testing.assert_allclose(gc.cpu().numpy(), wc, atol=2e-4)
    # without the exact flag the coordinate gradient is zero
    gz = _dne().altcorr_index_backward(f.cuda(), [lv.cuda() for lv in levels], coords.cuda(), ii.cuda(), jj.cuda(),
                                       grad.cuda(), 3, False)[2]
    assert float(gz.abs().max()) == 0.0


def test_altcorrblock_indexed_gradients_match_per_level_route():
    """AltCorrBlock: gradients (feature maps through the pooled pyramid, coordinates) of the
    indexed lookup equal those of the per-level on-the-fly route (the reference's checking route
    for the forward, tests/test_altcorr_indexed.py)."""
    from vipe_b200.droid_corr import AltCorrBlock, AltCorrIndex, CorrLayer

    g = torch.Generator().manual_seed(19)
    B, N, C, H, W, E = 1, 5, 64, 16, 32, 6
    fmaps0 = torch.randn(B, N, C, H, W, generator=g).cuda()
    ii = torch.tensor([0, 1, 2, 3, 0, 4], device="cuda")
    jj = torch.tensor([1, 2, 3, 4, 2, 2], device="cuda")
    yy, xx = torch.meshgrid(torch.arange(H), torch.arange(W), indexing="ij")
    coords0 = (torch.stack([xx, yy], -1).float()[None].repeat(B, E, 1, 1, 1)
               + 0.8 * torch.randn(B, E, H, W, 2, generator=g)).cuda()
    R = torch.randn(B, E, 4 * 49, H, W, generator=g).cuda()
    grads = []
    for route in ("indexed", "reference"):
        fm = fmaps0.clone().requires_grad_()
        co = coords0.clone().requires_grad_()
        AltCorrIndex.exact_coords_grad = CorrLayer.exact_coords_grad = True
        try:
            blk = AltCorrBlock(fm)
            cs = co.unsqueeze(-2)
            out = blk.corr_fn_indexed(cs, ii, jj) if route == "indexed" else blk.corr_fn_reference(cs, ii, jj)
            (out[..., 0] * R).sum().backward()
        finally:
            AltCorrIndex.exact_coords_grad = CorrLayer.exact_coords_grad = False
        grads.append((fm.grad, co.grad))
    (a1, ac), (b1, bc) = grads
    torch.testing.assert_close(a1, b1, atol=1e-4, rtol=1e-4)
    torch.testing.assert_close(ac, bc, atol=1e-4, rtol=1e-4)


@pytest.mark.parametrize("dtype,C,sigma,W", [(torch.float16, 128, 0.4, 64), (torch.bfloat16, 64, 6.0, 20),
                                             (torch.float16, 256, 1.0, 13), (torch.float32, 32, 1.0, 16)])
def test_altcorr_index_forward_paths(dtype, C, sigma, W):
    """Indexed lookup vs the FP64 oracle: 16-bit maps with C in {64, 128, 256} take the tensor-core
    union-box kernel (smooth coordinates: one box per 8 pixels; sigma = 6 px: boxes too large, one
    pass per pixel; W not a multiple of 8: partial warps); f32 maps the element kernel."""
    g = torch.Generator().manual_seed(21)
    B, Nf, H, M = 1, 4, 8, 3
    f = (torch.randn(B, Nf, H, W, C, generator=g) / C**0.5).to(dtype)
    levels = [f]
    for _ in range(3):
        t = levels[-1].float().permute(0, 1, 4, 2, 3).reshape(B * Nf, C, levels[-1].shape[2], levels[-1].shape[3])
        t = torch.nn.functional.avg_pool2d(t, 2, stride=2)
        levels.append(t.reshape(B, Nf, C, t.shape[-2], t.shape[-1]).permute(0, 1, 3, 4, 2).contiguous().to(dtype))
    ii, jj = torch.tensor([0, 1, 3]), torch.tensor([1, 2, 1])
    coords = _grid_coords(B * M, H, W, g, sigma).reshape(B, M, 2, H, W).permute(0, 1, 3, 4, 2).contiguous()
    coords[0, 0, 0, 0] = torch.tensor([1e9, -1e9])  # far away: zeros, and the box falls back to per-pixel passes
    out = _dne().altcorr_index_forward(f.cuda(), [lv.cuda() for lv in levels], coords.cuda(), ii.cuda(), jj.cuda(),
                                       3)[0]
    want = oc.altcorr_index_forward(f.double().numpy(), [lv.double().numpy() for lv in levels], coords.numpy(),
                                    ii.numpy(), jj.numpy(), 3)
    np.testing.assert_allclose(out.double().cpu().numpy(), want, atol=1e-4)


@pytest.mark.parametrize("levels", [1, 2, 3])
def test_volume_build_full_row_path_fewer_levels(levels):
    """64-wide 16-bit maps take the full-row TMA-store epilogue; with fewer than 4 levels only the
    requested levels are stored (and no level-3 pooling pass runs)."""
    from vipe_b200.corr_build import corr_volume_pyramid

    g = torch.Generator().manual_seed(22)
    num, C, H, W = 2, 128, 16, 64
    f1 = (torch.randn(num, C, H, W, generator=g) / np.sqrt(C) * 4).to(torch.bfloat16)
    f2 = (torch.randn(num, C, H, W, generator=g) / np.sqrt(C) * 4).to(torch.bfloat16)
    got = corr_volume_pyramid(f1.cuda(), f2.cuda(), levels, out_dtype=torch.float16)
    assert len(got) == levels
    want = oc.corr_pyramid(f1.double().numpy(), f2.double().numpy(), levels)
    for l, (a, w) in enumerate(zip(got, want)):
        a = a.cpu().double().numpy().reshape(w.shape)
        assert np.abs(a - w).max() <= 2e-3 * np.abs(w).max(), l
