"""FP64 numpy restatement of the correlation ops — TEST INFRASTRUCTURE ONLY.

Follows the reference:
  * CorrBlock.corr + pyramid  vipe/slam/networks/droid_net.py:56-69, 94-102
    (fmaps / 4, all-pairs dot over channels, avg_pool2d(2) over the target axes,
    floor sizes);
  * corr_index_forward / backward  csrc/droid_net_ext/correlation_kernels.cu:22-113
    (taps floor(x) - r + i, channel i * (2r+1) + j with i the x offset, bilinear
    weights from the fractional part, zeros outside);
  * altcorr_forward / backward / altcorr_index_forward
    csrc/droid_net_ext/altcorr_kernel.cu:26-366 (same taps on the fly; coords / 2^l
    per pyramid level; output f32 for the indexed form).
The reference's altcorr_backward leaves the coords gradient at zero
(altcorr_kernel.cu:440); `altcorr_backward(..., exact_coords=True)` here returns
the derivative of the bilinear weights instead.  `corr_index_coords_backward`
is that derivative for the volume lookup (the reference's CorrSampler returns
none, droid_net.py:40-45), and `corr_pyramid_backward` the feature-map gradient
of the pyramid that torch autograd forms in the reference (matmul and
avg_pool2d, droid_net.py:56-69, 94-102): every level gradient spread back to
level 0, then the two products with the other feature map.
"""

from __future__ import annotations

import numpy as np


def corr_volume(fmap1, fmap2):
    """(B, C, H, W) x2 -> (B, H, W, H, W): (fmap1/4)^T (fmap2/4)."""
    f1 = np.asarray(fmap1, np.float64) / 4.0
    f2 = np.asarray(fmap2, np.float64) / 4.0
    B, C, H, W = f1.shape
    v = np.einsum("bcp,bcq->bpq", f1.reshape(B, C, H * W), f2.reshape(B, C, H * W))
    return v.reshape(B, H, W, H, W)


def avg_pool2(v):
    """2x2 average pool over the last two axes (floor sizes)."""
    h, w = v.shape[-2] // 2, v.shape[-1] // 2
    v = v[..., : 2 * h, : 2 * w]
    return 0.25 * (v[..., 0::2, 0::2] + v[..., 1::2, 0::2] + v[..., 0::2, 1::2] + v[..., 1::2, 1::2])


def corr_pyramid(fmap1, fmap2, levels=4):
    v = corr_volume(fmap1, fmap2)
    out = [v]
    for _ in range(levels - 1):
        v = avg_pool2(v)
        out.append(v)
    return out


def _bilinear_from_taps(taps, x, y, r):
    """taps (..., rd+1, rd+1) indexed [i][j] (x offset i, y offset j) -> (..., rd, rd)."""
    dx = (x - np.floor(x))[..., None, None]
    dy = (y - np.floor(y))[..., None, None]
    return ((1 - dx) * (1 - dy) * taps[..., :-1, :-1] + dx * (1 - dy) * taps[..., 1:, :-1]
            + (1 - dx) * dy * taps[..., :-1, 1:] + dx * dy * taps[..., 1:, 1:])


def _tap_index(x, y, r):
    rd = 2 * r + 1
    off = np.arange(rd + 1)
    X = np.floor(x).astype(np.int64)[..., None, None] - r + off[:, None]
    Y = np.floor(y).astype(np.int64)[..., None, None] - r + off[None, :]
    X, Y = np.broadcast_arrays(X, Y)
    return X.copy(), Y.copy()


def corr_index_forward(volume, coords, r):
    """volume (B, h1, w1, h2, w2), coords (B, 2, h1, w1) -> (B, rd, rd, h1, w1)."""
    vol = np.asarray(volume, np.float64)
    c = np.asarray(coords, np.float64)
    B, h1, w1, h2, w2 = vol.shape
    x, y = c[:, 0], c[:, 1]
    X, Y = _tap_index(x, y, r)
    ok = (X >= 0) & (X < w2) & (Y >= 0) & (Y < h2)
    bb = np.arange(B)[:, None, None, None, None]
    pp = np.arange(h1)[None, :, None, None, None]
    qq = np.arange(w1)[None, None, :, None, None]
    taps = vol[bb, pp, qq, np.clip(Y, 0, h2 - 1), np.clip(X, 0, w2 - 1)] * ok
    out = _bilinear_from_taps(taps, x, y, r)  # (B, h1, w1, rd, rd)
    return out.transpose(0, 3, 4, 1, 2)


def corr_index_backward(volume_shape, coords, grad, r):
    c = np.asarray(coords, np.float64)
    g = np.asarray(grad, np.float64)
    B, h1, w1, h2, w2 = volume_shape
    rd = 2 * r + 1
    x, y = c[:, 0], c[:, 1]
    dx = x - np.floor(x)
    dy = y - np.floor(y)
    X, Y = _tap_index(x, y, r)
    gg = g.transpose(0, 3, 4, 1, 2)  # (B, h1, w1, rd, rd)
    tg = np.zeros((B, h1, w1, rd + 1, rd + 1))
    dxe, dye = dx[..., None, None], dy[..., None, None]
    tg[..., :-1, :-1] += gg * (1 - dxe) * (1 - dye)
    tg[..., 1:, :-1] += gg * dxe * (1 - dye)
    tg[..., :-1, 1:] += gg * (1 - dxe) * dye
    tg[..., 1:, 1:] += gg * dxe * dye
    out = np.zeros(volume_shape)
    ok = (X >= 0) & (X < w2) & (Y >= 0) & (Y < h2)
    for b in range(B):
        for p in range(h1):
            for q in range(w1):
                m = ok[b, p, q]
                out[b, p, q, Y[b, p, q][m], X[b, p, q][m]] = tg[b, p, q][m]
    return out


def corr_index_coords_backward(volume, coords, grad, r):
    """volume (B,h1,w1,h2,w2), coords (B,2,h1,w1), grad (B,rd,rd,h1,w1) -> (B,2,h1,w1)."""
    vol = np.asarray(volume, np.float64)
    c = np.asarray(coords, np.float64)
    g = np.asarray(grad, np.float64)
    B, h1, w1, h2, w2 = vol.shape
    x, y = c[:, 0], c[:, 1]
    dx = (x - np.floor(x))[..., None, None]
    dy = (y - np.floor(y))[..., None, None]
    X, Y = _tap_index(x, y, r)
    ok = (X >= 0) & (X < w2) & (Y >= 0) & (Y < h2)
    bb = np.arange(B)[:, None, None, None, None]
    pp = np.arange(h1)[None, :, None, None, None]
    qq = np.arange(w1)[None, None, :, None, None]
    t = vol[bb, pp, qq, np.clip(Y, 0, h2 - 1), np.clip(X, 0, w2 - 1)] * ok  # (B,h1,w1,rd+1,rd+1) [x off][y off]
    a00, a10, a01, a11 = t[..., :-1, :-1], t[..., 1:, :-1], t[..., :-1, 1:], t[..., 1:, 1:]
    ddx = (1 - dy) * (a10 - a00) + dy * (a11 - a01)
    ddy = (1 - dx) * (a01 - a00) + dx * (a11 - a10)
    gg = g.transpose(0, 3, 4, 1, 2)
    return np.stack([(gg * ddx).sum((-1, -2)), (gg * ddy).sum((-1, -2))], 1)


def corr_pyramid_backward(fmap1, fmap2, level_grads):
    """fmap1, fmap2 (B,C,H,W); level_grads[l] (B,H,W,H>>l,W>>l) (None: no gradient) -> (d fmap1, d fmap2)."""
    f1 = np.asarray(fmap1, np.float64)
    f2 = np.asarray(fmap2, np.float64)
    B, C, H, W = f1.shape
    g0 = np.zeros((B, H * W, H, W))
    for l, G in enumerate(level_grads):
        if G is None:
            continue
        G = np.asarray(G, np.float64).reshape(B, H * W, H >> l, W >> l)
        # adjoint of l average pools: each pooled value spread evenly over its 2^l x 2^l block
        g0 += np.repeat(np.repeat(G, 2**l, axis=2), 2**l, axis=3) / 4.0**l
    g0 = g0.reshape(B, H * W, H * W)
    d1 = np.einsum("bpq,bcq->bcp", g0, f2.reshape(B, C, H * W)) / 16.0
    d2 = np.einsum("bpq,bcp->bcq", g0, f1.reshape(B, C, H * W)) / 16.0
    return d1.reshape(B, C, H, W), d2.reshape(B, C, H, W)


def _window_dots(f1, f2, x, y, r):
    """f1 (H1,W1,C), f2 (H2,W2,C), x,y (H1,W1) -> taps (H1,W1,rd+1,rd+1)."""
    H2, W2, C = f2.shape
    X, Y = _tap_index(x, y, r)
    ok = (X >= 0) & (X < W2) & (Y >= 0) & (Y < H2)
    g = f2[np.clip(Y, 0, H2 - 1), np.clip(X, 0, W2 - 1)]  # (H1,W1,rd+1,rd+1,C)
    return np.einsum("hwc,hwijc->hwij", f1, g) * ok


def altcorr_forward(fmap1, fmap2, coords, r):
    """fmap1 (B,H1,W1,C), fmap2 (B,H2,W2,C), coords (B,S,H1,W1,2) -> (B,S,rd^2,H1,W1)."""
    f1 = np.asarray(fmap1, np.float64)
    f2 = np.asarray(fmap2, np.float64)
    c = np.asarray(coords, np.float64)
    B, S = c.shape[:2]
    rd = 2 * r + 1
    out = np.zeros((B, S, rd * rd) + c.shape[2:4])
    for b in range(B):
        for s in range(S):
            x, y = c[b, s, ..., 0], c[b, s, ..., 1]
            t = _window_dots(f1[b], f2[b], x, y, r)
            o = _bilinear_from_taps(t, x, y, r)  # (H1,W1,rd,rd)
            out[b, s] = o.reshape(o.shape[0], o.shape[1], rd * rd).transpose(2, 0, 1)
    return out


def altcorr_backward(fmap1, fmap2, coords, grad, r, exact_coords=False):
    f1 = np.asarray(fmap1, np.float64)
    f2 = np.asarray(fmap2, np.float64)
    c = np.asarray(coords, np.float64)
    g = np.asarray(grad, np.float64)
    B, S, H1, W1, _ = c.shape
    H2, W2, C = f2.shape[1:]
    rd = 2 * r + 1
    g1 = np.zeros_like(f1)
    g2 = np.zeros_like(f2)
    gc = np.zeros_like(c)
    for b in range(B):
        for s in range(S):
            x, y = c[b, s, ..., 0], c[b, s, ..., 1]
            dx = (x - np.floor(x))[..., None, None]
            dy = (y - np.floor(y))[..., None, None]
            gg = g[b, s].reshape(rd, rd, H1, W1).transpose(2, 3, 0, 1)
            tg = np.zeros((H1, W1, rd + 1, rd + 1))
            tg[..., :-1, :-1] += gg * (1 - dx) * (1 - dy)
            tg[..., 1:, :-1] += gg * dx * (1 - dy)
            tg[..., :-1, 1:] += gg * (1 - dx) * dy
            tg[..., 1:, 1:] += gg * dx * dy
            X, Y = _tap_index(x, y, r)
            ok = (X >= 0) & (X < W2) & (Y >= 0) & (Y < H2)
            tg = tg * ok
            Yc, Xc = np.clip(Y, 0, H2 - 1), np.clip(X, 0, W2 - 1)
            g1[b] += np.einsum("hwij,hwijc->hwc", tg, f2[b][Yc, Xc])
            np.add.at(g2[b], (Yc, Xc), tg[..., None] * f1[b][:, :, None, None, :])
            if exact_coords:
                t = _window_dots(f1[b], f2[b], x, y, r)
                a00, a10, a01, a11 = t[..., :-1, :-1], t[..., 1:, :-1], t[..., :-1, 1:], t[..., 1:, 1:]
                ddx = (1 - dy) * (a10 - a00) + dy * (a11 - a01)
                ddy = (1 - dx) * (a01 - a00) + dx * (a11 - a10)
                gc[b, s, ..., 0] = (gg * ddx).sum((-1, -2))
                gc[b, s, ..., 1] = (gg * ddy).sum((-1, -2))
    return g1, g2, gc


def altcorr_index_forward(fmap1, levels, coords, ii, jj, r):
    """fmap1 (B,Nf,H,W,C), levels[l] (B,Nf,Hl,Wl,C), coords (B,M,H,W,2) -> (B,M,L*rd^2,H,W)."""
    f1 = np.asarray(fmap1, np.float64)
    c = np.asarray(coords, np.float64)
    B, M, H, W, _ = c.shape
    rd = 2 * r + 1
    L = len(levels)
    out = np.zeros((B, M, L * rd * rd, H, W))
    for l, lv in enumerate(levels):
        f2 = np.asarray(lv, np.float64)
        for b in range(B):
            for m in range(M):
                x = c[b, m, ..., 0] / 2 ** l
                y = c[b, m, ..., 1] / 2 ** l
                t = _window_dots(f1[b, ii[m]], f2[b, jj[m]], x, y, r)
                o = _bilinear_from_taps(t, x, y, r)
                out[b, m, l * rd * rd:(l + 1) * rd * rd] = o.reshape(H, W, rd * rd).transpose(2, 0, 1)
    return out


def altcorr_index_backward(fmap1, levels, coords, ii, jj, grad, r, exact_coords=False):
    """Adjoint of altcorr_index_forward: -> (d fmap1, [d level], d coords), each edge and level
    the per-level altcorr_backward at coords / 2^l (coords gradient scaled back by 2^-l)."""
    f1 = np.asarray(fmap1, np.float64)
    c = np.asarray(coords, np.float64)
    g = np.asarray(grad, np.float64)
    B, M, H, W, _ = c.shape
    rd = 2 * r + 1
    g1 = np.zeros_like(f1)
    gl = [np.zeros(np.shape(lv)) for lv in levels]
    gc = np.zeros_like(c)
    for l, lv in enumerate(levels):
        f2 = np.asarray(lv, np.float64)
        for m in range(M):
            a, b, cc = altcorr_backward(f1[:, ii[m]], f2[:, jj[m]], c[:, m:m + 1] / 2 ** l,
                                        g[:, m:m + 1, l * rd * rd:(l + 1) * rd * rd], r, exact_coords=exact_coords)
            g1[:, ii[m]] += a
            gl[l][:, jj[m]] += b
            gc[:, m] += cc[:, 0] / 2 ** l
    return g1, gl, gc
