"""lietorch_ext on the GPU against the FP64 oracle (oracle/lie.py).

All 19 bound ops (reference csrc/lietorch_ext/lietorch.cpp:306-336) for SO3,
RxSO3, SE3, Sim3 in float64 (atol 1e-9) and float32 (atol 2e-4 on O(1)
values).  Inputs include non-unit quaternions (normalised on load, as in the
reference), small-angle tangents (series branches) and a batch of 0.
"""

import numpy as np
import pytest
import torch

import oracle.lie as L

pytestmark = pytest.mark.gpu

GROUPS = [1, 2, 3, 4]
DTYPES = [torch.float64, torch.float32]
TOL = {torch.float64: 1e-9, torch.float32: 2e-4}


def _lt():
    from vipe_b200.ext import lietorch_ext

    return lietorch_ext


def _inputs(gid, B, seed, dtype):
    rng = np.random.default_rng(seed)
    N, K = L.DIMS[gid]
    a = rng.normal(0, 0.5, (B, K))
    a[: B // 8] *= 1e-7  # small-angle branch
    X = np.stack([L.exp(gid, r).data() for r in rng.normal(0, 0.6, (B, K))])
    qs = slice(0, 4) if gid in (1, 2) else slice(3, 7)
    X[:, qs] *= rng.uniform(0.7, 1.3, (B, 1))  # non-unit quaternions
    Y = np.stack([L.exp(gid, r).data() for r in rng.normal(0, 0.6, (B, K))])
    p3 = rng.normal(0, 1, (B, 3))
    p4 = np.concatenate([p3, rng.uniform(0.1, 1, (B, 1))], 1)
    gN = rng.normal(0, 1, (B, N))
    gK = rng.normal(0, 1, (B, K))
    g3 = rng.normal(0, 1, (B, 3))
    g4 = rng.normal(0, 1, (B, 4))
    t = lambda x: torch.tensor(x, dtype=dtype, device="cuda")
    return {k: (v, t(v)) for k, v in dict(a=a, X=X, Y=Y, p3=p3, p4=p4, gN=gN, gK=gK, g3=g3, g4=g4).items()}


def _cmp(got, want, dtype, scale=1.0):
    got = got.detach().cpu().double().numpy()
    np.testing.assert_allclose(got, want, atol=TOL[dtype] * scale, rtol=TOL[dtype])


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("gid", GROUPS)
def test_forward_ops(gid, dtype):
    lt = _lt()
    I = _inputs(gid, 64, 100 + gid, dtype)
    X = I["X"]
    _cmp(lt.expm(gid, I["a"][1]), L.expm(gid, I["a"][0]), dtype)
    _cmp(lt.logm(gid, X[1]), L.logm(gid, X[0]), dtype, 10)
    _cmp(lt.inv(gid, X[1]), L.inv(gid, X[0]), dtype)
    _cmp(lt.mul(gid, X[1], I["Y"][1]), L.mul(gid, X[0], I["Y"][0]), dtype)
    _cmp(lt.adj(gid, X[1], I["a"][1]), L.adj(gid, X[0], I["a"][0]), dtype)
    _cmp(lt.adjT(gid, X[1], I["a"][1]), L.adjT(gid, X[0], I["a"][0]), dtype)
    _cmp(lt.act(gid, X[1], I["p3"][1]), L.act(gid, X[0], I["p3"][0]), dtype)
    _cmp(lt.act4(gid, X[1], I["p4"][1]), L.act4(gid, X[0], I["p4"][0]), dtype)
    _cmp(lt.as_matrix(gid, X[1]), L.as_matrix(gid, X[0]), dtype)
    _cmp(lt.projector(gid, X[1]), L.projector(gid, X[0]), dtype)
    _cmp(lt.Jinv(gid, X[1], I["a"][1]), L.Jinv(gid, X[0], I["a"][0]), dtype, 10)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("gid", GROUPS)
def test_backward_ops(gid, dtype):
    lt = _lt()
    I = _inputs(gid, 64, 200 + gid, dtype)
    X, Y, a = I["X"], I["Y"], I["a"]
    (da,) = lt.expm_backward(gid, I["gN"][1], a[1])
    _cmp(da, L.expm_backward(gid, I["gN"][0], a[0]), dtype)
    (dX,) = lt.logm_backward(gid, I["gK"][1], X[1])
    _cmp(dX, L.logm_backward(gid, I["gK"][0], X[0]), dtype, 10)
    (dX,) = lt.inv_backward(gid, I["gN"][1], X[1])
    _cmp(dX, L.inv_backward(gid, I["gN"][0], X[0]), dtype)
    dX, dY = lt.mul_backward(gid, I["gN"][1], X[1], Y[1])
    wX, wY = L.mul_backward(gid, I["gN"][0], X[0], Y[0])
    _cmp(dX, wX, dtype)
    _cmp(dY, wY, dtype)
    for fn in ("adj_backward", "adjT_backward"):
        dX, da = getattr(lt, fn)(gid, I["gK"][1], X[1], a[1])
        wX, wa = getattr(L, fn)(gid, I["gK"][0], X[0], a[0])
        _cmp(dX, wX, dtype)
        _cmp(da, wa, dtype)
    dX, dp = lt.act_backward(gid, I["g3"][1], X[1], I["p3"][1])
    wX, wp = L.act_backward(gid, I["g3"][0], X[0], I["p3"][0])
    _cmp(dX, wX, dtype)
    _cmp(dp, wp, dtype)
    dX, dp = lt.act4_backward(gid, I["g4"][1], X[1], I["p4"][1])
    wX, wp = L.act4_backward(gid, I["g4"][0], X[0], I["p4"][0])
    _cmp(dX, wX, dtype)
    _cmp(dp, wp, dtype)


def test_empty_batch_and_errors():
    lt = _lt()
    X = torch.zeros(0, 7, device="cuda")
    assert lt.inv(3, X).shape == (0, 7)
    with pytest.raises(RuntimeError):
        lt.inv(5, torch.zeros(2, 7, device="cuda"))
    with pytest.raises(RuntimeError):
        lt.inv(3, torch.zeros(2, 7, device="cuda", dtype=torch.float16))
    with pytest.raises(RuntimeError):
        lt.inv(3, torch.zeros(2, 7))  # CPU tensor: no CPU path
