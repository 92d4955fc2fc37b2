"""Seeded synthetic dense-CRF workloads.

The reference measures on its own ``data/img.bmp`` + ``data/img.c_unary`` and on
MSRC-style images; neither is shipped here, so every benchmark and parity case
uses this generator instead, with the shapes and value distributions of the
reference's example (``src/example_inference.cpp:15-88``):

* an RGB image made of ``n_seeds`` piecewise-constant Voronoi regions (uniform
  seed positions, uniform seed colours) plus Gaussian noise of s.d. ``noise``,
  rounded and clamped to uint8, stored pixel-major ``[H][W][3]`` exactly like
  the buffer ``DenseCRF2D::addPairwiseBilateral`` reads
  (``src/densecrf.cpp:179-190``);
* unaries ``U = -log softmax(logits)`` with ``logits ~ N(0, 1)`` per
  (pixel, label) and ``+boost`` on the label assigned to the pixel's region,
  float32, laid out ``[N][L]`` (label fastest), which is the memory order of
  the reference's column-major ``MatrixXf(L, N)``.
"""
from __future__ import annotations

import numpy as np

GAUSSIAN = dict(sxy=3.0, w=3.0)
BILATERAL = dict(sxy=50.0, srgb=15.0, w=5.0)


def voronoi_image(W: int, H: int, seed: int, n_seeds: int = 40, noise: float = 8.0,
                  n_labels: int = 21):
    """Returns ``(rgb uint8 [H*W*3], region_label int32 [H*W])``."""
    rng = np.random.default_rng(seed)
    sx = rng.uniform(0, W, n_seeds)
    sy = rng.uniform(0, H, n_seeds)
    col = rng.uniform(0, 256, (n_seeds, 3))
    lab = rng.integers(0, n_labels, n_seeds)
    ys, xs = np.mgrid[0:H, 0:W]
    best = np.full((H, W), np.inf)
    owner = np.zeros((H, W), np.int64)
    for s in range(n_seeds):
        dd = (xs - sx[s]) ** 2 + (ys - sy[s]) ** 2
        m = dd < best
        best[m] = dd[m]
        owner[m] = s
    img = col[owner] + rng.normal(0.0, noise, (H, W, 3))
    img = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    return np.ascontiguousarray(img.reshape(-1)), lab[owner].reshape(-1).astype(np.int32)


def unaries(region_label: np.ndarray, n_labels: int, seed: int, boost: float = 2.0):
    """``-log softmax`` unaries, float32 ``[N][L]``."""
    rng = np.random.default_rng(seed + 7919)
    N = region_label.shape[0]
    logits = rng.normal(0.0, 1.0, (N, n_labels))
    logits[np.arange(N), region_label] += boost
    logits -= logits.max(axis=1, keepdims=True)
    lse = np.log(np.exp(logits).sum(axis=1, keepdims=True))
    return np.ascontiguousarray((lse - logits).astype(np.float32))


def make_image(W: int, H: int, L: int = 21, seed: int = 0):
    """One synthetic CRF instance: ``dict(W, H, L, rgb, unary)``."""
    rgb, reg = voronoi_image(W, H, seed, n_labels=L)
    return dict(W=W, H=H, L=L, rgb=rgb, unary=unaries(reg, L, seed))


def gaussian_features(W: int, H: int, sx: float, sy: float):
    """Features of ``DenseCRF2D::addPairwiseGaussian`` (``src/densecrf.cpp:170-178``),
    float32 ``[N][2]``: ``(x/sx, y/sy)`` computed in float like the reference."""
    ys, xs = np.mgrid[0:H, 0:W]
    f = np.empty((H * W, 2), np.float32)
    f[:, 0] = xs.reshape(-1).astype(np.float32) / np.float32(sx)
    f[:, 1] = ys.reshape(-1).astype(np.float32) / np.float32(sy)
    return f


def bilateral_features(W: int, H: int, sx: float, sy: float, sr: float, sg: float, sb: float,
                       rgb: np.ndarray):
    """Features of ``DenseCRF2D::addPairwiseBilateral`` (``src/densecrf.cpp:179-190``),
    float32 ``[N][5]``."""
    f = np.empty((H * W, 5), np.float32)
    g = gaussian_features(W, H, sx, sy)
    f[:, :2] = g
    px = rgb.reshape(-1, 3).astype(np.float32)
    f[:, 2] = px[:, 0] / np.float32(sr)
    f[:, 3] = px[:, 1] / np.float32(sg)
    f[:, 4] = px[:, 2] / np.float32(sb)
    return f


def batch_sizes(n: int, seed: int, lo=(240, 320), hi=(500, 500)):
    """Uneven image sizes ``[(W, H)]`` of the batched workload: H ~ U[240, 500],
    W ~ U[320, 500] (integers, seeded)."""
    rng = np.random.default_rng(seed)
    Hs = rng.integers(lo[0], hi[0] + 1, n)
    Ws = rng.integers(lo[1], hi[1] + 1, n)
    return [(int(w), int(h)) for w, h in zip(Ws, Hs)]


def superpixels(rgb: np.ndarray, W: int, H: int, spacing: int, seed: int, colour_weight: float = 20.0):
    """A seeded superpixel segmentation standing in for the reference's EDISON
    mean-shift (``addSuperPixel``): jittered grid seeds ``spacing`` pixels
    apart, each pixel joined to the nearest of its 3x3 neighbouring seeds in
    (x, y, rgb) with colour distances scaled by ``spacing / colour_weight``.
    Returns ``region int32 [H*W]``, ids ``0 .. R-1`` in first-pixel order."""
    rng = np.random.default_rng(seed)
    gx, gy = (W + spacing - 1) // spacing, (H + spacing - 1) // spacing
    sx = (np.arange(gx) + 0.5)[None, :] * spacing + rng.uniform(-0.25, 0.25, (gy, gx)) * spacing
    sy = (np.arange(gy) + 0.5)[:, None] * spacing + rng.uniform(-0.25, 0.25, (gy, gx)) * spacing
    sx = np.clip(sx, 0, W - 1)
    sy = np.clip(sy, 0, H - 1)
    img = rgb.reshape(H, W, 3).astype(np.float64)
    scol = img[sy.astype(int), sx.astype(int)]
    ys, xs = np.mgrid[0:H, 0:W]
    cx, cy = xs // spacing, ys // spacing
    best = np.full((H, W), np.inf)
    owner = np.zeros((H, W), np.int64)
    for oy in (-1, 0, 1):
        for ox in (-1, 0, 1):
            tx, ty = cx + ox, cy + oy
            ok = (tx >= 0) & (tx < gx) & (ty >= 0) & (ty < gy)
            txc, tyc = np.clip(tx, 0, gx - 1), np.clip(ty, 0, gy - 1)
            dxy = ((xs - sx[tyc, txc]) ** 2 + (ys - sy[tyc, txc]) ** 2) / spacing ** 2
            dc = ((img - scol[tyc, txc]) ** 2).sum(-1) / colour_weight ** 2
            dd = np.where(ok, dxy + dc, np.inf)
            m = dd < best
            best[m] = dd[m]
            owner[m] = (tyc * gx + txc)[m]
    _, first, inv = np.unique(owner.reshape(-1), return_index=True, return_inverse=True)
    order = np.argsort(np.argsort(first))  # renumber by first pixel
    return order[inv].astype(np.int32)


def clique_state(rgb: np.ndarray, region: np.ndarray, constant: float, normaliser: float,
                 min_size: int = 500, max_size: int = 2000):
    """The clique state ``addSuperPixel`` derives from a segmentation
    (``src/densecrf.cpp:212-247``): per region its pixel ids, the weight
    ``constant * exp(-sum (grey - mean)^2 / (normaliser * count))`` with the
    reference's grey level ``0.2989 img[i] + 0.5870 img[i+1] + 0.1140 img[i+2]``
    (byte offsets i, i+1, i+2, as the reference reads them), and ``constant``.
    Evaluated in float64, rounded to float32.  Only regions of
    ``min_size .. max_size`` pixels are kept.  Returns
    ``(offsets, idx, exp_weight, constants)``."""
    N = region.shape[0]
    b = rgb.astype(np.float64)
    i = np.arange(N)
    grey = 0.2989 * b[i] + 0.5870 * b[i + 1] + 0.1140 * b[i + 2]
    R = int(region.max()) + 1
    cnt = np.bincount(region, minlength=R).astype(np.float64)
    mean = np.bincount(region, grey, R) / cnt
    sd = np.bincount(region, (grey - mean[region]) ** 2, R) / (normaliser * cnt)
    keep = np.nonzero((cnt >= min_size) & (cnt <= max_size))[0]
    order = np.argsort(region, kind="stable")
    starts = np.concatenate([[0], np.cumsum(cnt.astype(np.int64))])
    idx = np.concatenate([order[starts[r]:starts[r + 1]] for r in keep]).astype(np.int32) if len(keep) else \
        np.zeros(0, np.int32)
    offsets = np.concatenate([[0], np.cumsum(cnt[keep].astype(np.int64))]).astype(np.int32)
    expw = (constant * np.exp(-sd[keep])).astype(np.float32)
    consts = np.full(len(keep), constant, np.float32)
    return offsets, idx, expw, consts


def cliques_three_scales(img: dict, constant: float, normaliser: float, seed: int = 0):
    """Cliques of three superpixel scales (spacings 24 / 32 / 40 pixels, the
    stand-ins for mean-shift spatial radii 8 / 16 / 32), concatenated as
    repeated ``addSuperPixel`` calls concatenate them."""
    W, H, rgb = img["W"], img["H"], img["rgb"]
    parts = [clique_state(rgb, superpixels(rgb, W, H, sp, seed + k), constant, normaliser)
             for k, sp in enumerate((24, 32, 40))]
    offs, idx, ew, cs = [np.zeros(1, np.int32)], [], [], []
    base = 0
    for o, i, e, c in parts:
        offs.append(o[1:] + base)
        base += int(o[-1])
        idx.append(i)
        ew.append(e)
        cs.append(c)
    return (np.concatenate(offs).astype(np.int32), np.concatenate(idx), np.concatenate(ew), np.concatenate(cs))
