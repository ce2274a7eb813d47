"""CPU checks of the correlation oracle (oracle/corr.py).

Pins: (1) the materialised-volume route (CorrBlock.corr + corr_index) and the
on-the-fly route (altcorr) give the same lookup — the property the reference's
tests/test_altcorr_indexed.py checks between its indexed and per-level kernels;
(2) backward ops are the adjoints of the forward ops (<g, F(x)> = <F^T g, x>);
(3) the exact coords gradient matches central differences.
"""

import numpy as np
import pytest

import oracle.corr as oc


def _coords(B, H, W, rng, sigma=1.5):
    yy, xx = np.meshgrid(np.arange(H), np.arange(W), indexing="ij")
    return np.stack([xx, yy], 0)[None].repeat(B, 0) + rng.normal(0, sigma, (B, 2, H, W))


def test_volume_and_onthefly_routes_agree():
    rng = np.random.default_rng(1)
    B, C, H, W = 2, 16, 8, 8
    f1, f2 = rng.normal(size=(B, C, H, W)), rng.normal(size=(B, C, H, W))
    pyr = oc.corr_pyramid(f1, f2, 3)
    coords = _coords(B, H, W, rng)
    c5 = coords.transpose(0, 2, 3, 1)[:, None]
    # pyramid level l of the volume equals altcorr against the pooled fmap2 at coords / 2^l
    g1 = f1.transpose(0, 2, 3, 1) / 4
    g2 = f2 / 4
    for l, vol in enumerate(pyr):
        a = oc.corr_index_forward(vol, coords / 2 ** l, 3).reshape(B, 49, H, W)
        f2l = g2
        for _ in range(l):
            f2l = oc.avg_pool2(f2l)
        b = oc.altcorr_forward(g1, f2l.transpose(0, 2, 3, 1), c5 / 2 ** l, 3)[:, 0]
        np.testing.assert_allclose(a, b, atol=1e-12)


def test_indexed_matches_per_level():
    rng = np.random.default_rng(2)
    B, Nf, H, W, C = 1, 4, 8, 8, 8
    f = rng.normal(size=(B, Nf, H, W, C))
    levels = [f]
    for _ in range(2):
        t = levels[-1].transpose(0, 1, 4, 2, 3)
        levels.append(oc.avg_pool2(t).transpose(0, 1, 3, 4, 2))
    ii, jj = np.array([0, 1, 2]), np.array([1, 2, 3])
    coords = _coords(B * 3, H, W, rng).reshape(B, 3, 2, H, W).transpose(0, 1, 3, 4, 2)
    out = oc.altcorr_index_forward(f, levels, coords, ii, jj, 3)
    for l, lv in enumerate(levels):
        for m in range(3):
            ref = oc.altcorr_forward(f[:, ii[m]], lv[:, jj[m]], coords[:, m:m + 1] / 2 ** l, 3)[:, 0]
            np.testing.assert_allclose(out[:, m, l * 49:(l + 1) * 49], ref, atol=1e-12)


def test_backward_is_adjoint():
    rng = np.random.default_rng(3)
    B, H, W, C = 1, 6, 7, 8
    f1, f2 = rng.normal(size=(B, H, W, C)), rng.normal(size=(B, H, W, C))
    coords = _coords(B, H, W, rng).transpose(0, 2, 3, 1)[:, None]
    g = rng.normal(size=(B, 1, 49, H, W))
    g1, g2, _ = oc.altcorr_backward(f1, f2, coords, g, 3)
    d1, d2 = rng.normal(size=f1.shape), rng.normal(size=f2.shape)
    h = 1e-6
    lhs = (g * (oc.altcorr_forward(f1 + h * d1, f2 + h * d2, coords, 3) - oc.altcorr_forward(f1, f2, coords, 3))).sum() / h
    rhs = (g1 * d1).sum() + (g2 * d2).sum()
    assert abs(lhs - rhs) < 1e-4 * max(1.0, abs(rhs))
    # volume route
    vol = rng.normal(size=(B, H, W, H, W))
    c4 = coords[:, 0].transpose(0, 3, 1, 2)
    gv = rng.normal(size=(B, 7, 7, H, W))
    dvol = oc.corr_index_backward(vol.shape, c4, gv, 3)
    dv = rng.normal(size=vol.shape)
    lhs = (gv * oc.corr_index_forward(dv, c4, 3)).sum()
    np.testing.assert_allclose(lhs, (dvol * dv).sum(), rtol=1e-10)


def test_exact_coords_gradient_matches_fd():
    rng = np.random.default_rng(4)
    B, H, W, C = 1, 5, 6, 4
    f1, f2 = rng.normal(size=(B, H, W, C)), rng.normal(size=(B, H, W, C))
    coords = _coords(B, H, W, rng).transpose(0, 2, 3, 1)[:, None]
    coords = np.floor(coords) + np.clip(coords - np.floor(coords), 0.05, 0.95)  # away from cell borders
    g = rng.normal(size=(B, 1, 49, H, W))
    _, _, gc = oc.altcorr_backward(f1, f2, coords, g, 3, exact_coords=True)
    h = 1e-6
    for k in range(2):
        d = np.zeros_like(coords)
        d[..., k] = h
        num = (g * (oc.altcorr_forward(f1, f2, coords + d, 3) - oc.altcorr_forward(f1, f2, coords - d, 3))).sum(2) / (2 * h)
        np.testing.assert_allclose(gc[..., k], num, atol=1e-6)


def test_volume_coords_gradient_matches_fd():
    rng = np.random.default_rng(5)
    B, H, W = 2, 5, 6
    vol = rng.normal(size=(B, H, W, H, W))
    coords = _coords(B, H, W, rng)
    coords = np.floor(coords) + np.clip(coords - np.floor(coords), 0.05, 0.95)  # away from cell borders
    coords[0, :, 0, :2] -= 6.0  # some windows partly off the map
    g = rng.normal(size=(B, 7, 7, H, W))
    gc = oc.corr_index_coords_backward(vol, coords, g, 3)
    h = 1e-6
    for k in range(2):
        d = np.zeros_like(coords)
        d[:, k] = h
        num = (g * (oc.corr_index_forward(vol, coords + d, 3) - oc.corr_index_forward(vol, coords - d, 3))).sum(
            (1, 2)) / (2 * h)
        np.testing.assert_allclose(gc[:, k], num, atol=1e-6)


def test_pyramid_backward_is_adjoint():
    # <G, d pyramid(f1, f2)[d1, d2]> = <d fmap1, d1> + <d fmap2, d2> (the pyramid is bilinear:
    # its directional derivative is pyramid(d1, f2) + pyramid(f1, d2))
    rng = np.random.default_rng(6)
    B, C, H, W = 2, 6, 8, 8
    f1, f2 = rng.normal(size=(B, C, H, W)), rng.normal(size=(B, C, H, W))
    G = [rng.normal(size=(B, H, W, H >> l, W >> l)) for l in range(4)]
    G[2] = None  # a level without gradient
    g1, g2 = oc.corr_pyramid_backward(f1, f2, G)
    d1, d2 = rng.normal(size=f1.shape), rng.normal(size=f2.shape)
    pa, pb = oc.corr_pyramid(d1, f2, 4), oc.corr_pyramid(f1, d2, 4)
    lhs = sum((Gl * (a + b)).sum() for Gl, a, b in zip(G, pa, pb) if Gl is not None)
    np.testing.assert_allclose(lhs, (g1 * d1).sum() + (g2 * d2).sum(), rtol=1e-10)


def test_indexed_backward_is_adjoint():
    rng = np.random.default_rng(7)
    B, Nf, H, W, C = 1, 3, 8, 8, 4
    f = rng.normal(size=(B, Nf, H, W, C))
    levels = [f, rng.normal(size=(B, Nf, H // 2, W // 2, C))]
    ii, jj = np.array([0, 1, 0, 2]), np.array([1, 2, 2, 2])
    coords = _coords(B * 4, H, W, rng).reshape(B, 4, 2, H, W).transpose(0, 1, 3, 4, 2)
    coords = np.floor(coords) + np.clip(coords - np.floor(coords), 0.05, 0.95)
    g = rng.normal(size=(B, 4, 2 * 49, H, W))
    g1, gl, gc = oc.altcorr_index_backward(f, levels, coords, ii, jj, g, 3, exact_coords=True)
    d1 = rng.normal(size=f.shape)
    dl = [rng.normal(size=lv.shape) for lv in levels]
    h = 1e-6
    up = oc.altcorr_index_forward(f + h * d1, [lv + h * d for lv, d in zip(levels, dl)], coords, ii, jj, 3)
    dn = oc.altcorr_index_forward(f - h * d1, [lv - h * d for lv, d in zip(levels, dl)], coords, ii, jj, 3)
    lhs = (g * (up - dn)).sum() / (2 * h)
    rhs = (g1 * d1).sum() + sum((a * b).sum() for a, b in zip(gl, dl))
    np.testing.assert_allclose(lhs, rhs, rtol=1e-6)
    dc = rng.normal(size=coords.shape)
    up = oc.altcorr_index_forward(f, levels, coords + h * dc, ii, jj, 3)
    dn = oc.altcorr_index_forward(f, levels, coords - h * dc, ii, jj, 3)
    np.testing.assert_allclose((g * (up - dn)).sum() / (2 * h), (gc * dc).sum(), rtol=1e-6)
