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
