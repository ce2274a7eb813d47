"""vipe_b200's corr_ext (spatial correlation sampler) against the reference's own corr_ext.

The reference module (csrc/corr_ext/{correlation.cpp, correlation_sampler.cpp,
correlation_cuda_kernel.cu}) is compiled unchanged by oracle/build_ref.py into
oracle/_ref/ and run here on the same inputs: its CUDA path on GPU tensors, its CPU
loop (correlation.cpp) on CPU tensors.

* exact cases: small-integer maps make every sum exact in both implementations (the
  reference accumulates in the map type), so outputs and gradients compare with atol 0;
* the AOT tracker's configuration (kernel 1, a 15 x 15 patch with patch dilation 1 or 2,
  attention.py:174-181) and general ones (3 x 3 kernels, padding, dilation, stride, even
  patches);
* the backward is held to the reference's CUDA backward where that is the adjoint of its
  forward (kernel size 1, odd patches) and to its CPU backward (the exact adjoint of the
  CPU forward, which equals the GPU forward for odd patches) in FP64 elsewhere.
"""

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import build_ref

    return build_ref.load("ref_corr_ext")


def _ours():
    from vipe_b200.ext import corr_ext

    return corr_ext


def _ints(shape, gen, lo=-2, hi=3):
    return torch.randint(lo, hi, shape, generator=gen).float()


# (kH, kW, patchH, patchW, padH, padW, dilH, dilW, dpH, dpW, dH, dW)
AOT1 = (1, 1, 15, 15, 0, 0, 1, 1, 1, 1, 1, 1)
AOT2 = (1, 1, 15, 15, 0, 0, 1, 1, 2, 2, 1, 1)
GENERAL = (3, 3, 5, 7, 1, 2, 2, 1, 2, 1, 2, 1)
EVEN = (1, 1, 4, 6, 0, 0, 1, 1, 1, 2, 1, 1)


@pytest.mark.parametrize("cfg", [AOT1, AOT2, GENERAL, EVEN], ids=["aot", "aot_dil2", "general", "even_patch"])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float16, torch.bfloat16])
def test_forward_bit_exact_vs_reference_gpu(ref, cfg, dtype):
    g = torch.Generator().manual_seed(40)
    N, C, H, W = 3, 32, 30, 54
    lo, hi = (-2, 3) if dtype == torch.float32 else (-1, 2)  # FP16 / BF16 sums of <= 32*9 small products stay exact
    a = _ints((N, C, H, W), g, lo, hi).to(dtype).cuda()
    b = _ints((N, C, H, W), g, lo, hi).to(dtype).cuda()
    want = ref.forward(a, b, *cfg)
    got = _ours().forward(a, b, *cfg)
    assert got.shape == want.shape and got.dtype == want.dtype
    torch.testing.assert_close(got, want, atol=0, rtol=0)


@pytest.mark.parametrize("cfg", [AOT1, AOT2], ids=["aot", "aot_dil2"])
def test_backward_bit_exact_vs_reference_gpu(ref, cfg):
    g = torch.Generator().manual_seed(41)
    N, C, H, W = 2, 32, 24, 40
    a = _ints((N, C, H, W), g).cuda()
    b = _ints((N, C, H, W), g).cuda()
    out = ref.forward(a, b, *cfg)
    go = _ints(tuple(out.shape), g).cuda()
    w1, w2 = ref.backward(a, b, go, *cfg)
    g1, g2 = _ours().backward(a, b, go, *cfg)
    torch.testing.assert_close(g1, w1, atol=0, rtol=0)
    torch.testing.assert_close(g2, w2, atol=0, rtol=0)


@pytest.mark.parametrize("cfg", [AOT2, GENERAL], ids=["aot_dil2", "general"])
def test_forward_and_backward_vs_reference_cpu_fp64(ref, cfg):
    """FP64 Gaussian maps: the reference's CPU loop (forward and its exact adjoint) against
    vipe_b200 on the GPU, within 1e-12 relative."""
    g = torch.Generator().manual_seed(42)
    N, C, H, W = 2, 16, 20, 33
    a = torch.randn(N, C, H, W, generator=g, dtype=torch.float64)
    b = torch.randn(N, C, H, W, generator=g, dtype=torch.float64)
    want = ref.forward(a, b, *cfg)
    got = _ours().forward(a.cuda(), b.cuda(), *cfg).cpu()
    torch.testing.assert_close(got, want, atol=1e-12 * want.abs().max().item(), rtol=0)
    go = torch.randn(tuple(want.shape), generator=g, dtype=torch.float64)
    w1, w2 = ref.backward(a, b, go, *cfg)
    g1, g2 = _ours().backward(a.cuda(), b.cuda(), go.cuda(), *cfg)
    torch.testing.assert_close(g1.cpu(), w1, atol=1e-12 * w1.abs().max().item(), rtol=0)
    torch.testing.assert_close(g2.cpu(), w2, atol=1e-12 * w2.abs().max().item(), rtol=0)


@pytest.mark.parametrize("dtype,tol", [(torch.float32, 1e-5), (torch.float16, 2e-2), (torch.bfloat16, 1e-1)])
def test_forward_float_vs_reference_gpu(ref, dtype, tol):
    """Gaussian maps of unit scale, AOT configuration: FP32 within 1e-5 of the largest output;
    FP16 / BF16 within a few ulps (the reference sums 32 channels in the map type, vipe_b200 in
    FP32 with one rounding)."""
    g = torch.Generator().manual_seed(43)
    N, C, H, W = 4, 32, 30, 54
    a = (torch.randn(N, C, H, W, generator=g) / C**0.5).to(dtype).cuda()
    b = torch.randn(N, C, H, W, generator=g).to(dtype).cuda()
    want = ref.forward(a, b, *AOT2).float()
    got = _ours().forward(a, b, *AOT2).float()
    assert (got - want).abs().max() <= tol * want.abs().max()
