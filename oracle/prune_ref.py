"""NumPy restatement of the Speedy-Splat pruning scores
(photara/src/splat/rasterizer.cu:93-146, CudaRasterizer::pruning_scores
:450-490), in float64 over the CPU oracle's forward (draw list, per-tile
ranges, projected Gaussians, per-pixel last blended entry, rendered image).

TEST INFRASTRUCTURE ONLY: the checker for the library's pruning-score
kernel, used by tests/; never by the product.
"""
from __future__ import annotations

import numpy as np

TILE = 16
ALPHA_FLOOR = 1.0 / 255.0


def pixel_terms(ids, px, py, mean2d, conic, rgb, image_rgb, alpha_clip):
    """One pixel's walk: (Gaussian, derivative, per-channel derivative) for
    every blended entry of `ids` (already cut at the pixel's last entry)."""
    residual = float(np.sum(image_rgb))
    residual_rgb = np.array(image_rgb, np.float64)
    T = 1.0
    out = []
    for g in ids:
        dx = float(mean2d[g, 0]) - px
        dy = float(mean2d[g, 1]) - py
        co = conic[g].astype(np.float64)
        power = -0.5 * (co[0] * dx * dx + co[2] * dy * dy) - co[1] * dx * dy
        if power > 0:
            continue
        alpha = min(alpha_clip, co[3] * np.exp(power))
        if alpha < ALPHA_FLOOR:
            continue
        c = rgb[g, :3].astype(np.float64)
        residual -= T * alpha * c.sum()
        deriv = co[3] * (T * c.sum() - residual / (1 - alpha))
        residual_rgb -= T * alpha * c
        per = alpha * (T * c - residual_rgb / (1 - alpha))
        out.append((int(g), deriv, per))
        T *= 1 - alpha
    return out


def pruning_scores(fwd, width, height, n, alpha_clip=0.99, gaussian_pop=False):
    """Scores [n] from an oracle.cpu.render result (keys values, ranges,
    mean2d, conic, rgb, last, color): each tile's pixels walk its draw list
    together (vectorised over the pixels, in draw order)."""
    scores = np.zeros(n, np.float64)
    gx = (width + TILE - 1) // TILE
    image = fwd["color"].reshape(3, -1).astype(np.float64)
    last = fwd["last"].astype(np.int64)
    vals = fwd["values"].astype(np.int64)
    mean2d = fwd["mean2d"].astype(np.float64)
    conic = fwd["conic"].astype(np.float64)
    rgb = fwd["rgb"][:, :3].astype(np.float64)
    for t, (r0, r1) in enumerate(fwd["ranges"]):
        r0, r1 = int(r0), int(r1)
        if r1 <= r0:
            continue
        tx, ty = t % gx, t // gx
        ys, xs = np.mgrid[ty * TILE:min((ty + 1) * TILE, height),
                          tx * TILE:min((tx + 1) * TILE, width)]
        xs, ys = xs.ravel().astype(np.float64), ys.ravel().astype(np.float64)
        pix = (ys * width + xs).astype(np.int64)
        lim = np.minimum(r1 - r0, last[pix])
        residual = image[:, pix].sum(0)
        residual_rgb = image[:, pix].copy()
        T = np.ones(len(pix))
        for j in range(int(lim.max(initial=0))):
            g = vals[r0 + j]
            dx = mean2d[g, 0] - xs
            dy = mean2d[g, 1] - ys
            co = conic[g]
            power = -0.5 * (co[0] * dx * dx + co[2] * dy * dy) - co[1] * dx * dy
            alpha = np.minimum(alpha_clip, co[3] * np.exp(np.minimum(power, 0.0)))
            live = (j < lim) & ~(power > 0) & ~(alpha < ALPHA_FLOOR)
            c = rgb[g]
            residual = np.where(live, residual - T * alpha * c.sum(), residual)
            deriv = co[3] * (T * c.sum() - residual / (1 - alpha))
            residual_rgb = np.where(live, residual_rgb - T * alpha * c[:, None], residual_rgb)
            per = alpha * (T * c[:, None] - residual_rgb / (1 - alpha))
            value = (per * per).sum(0) if gaussian_pop else deriv * deriv
            scores[g] += float(value[live].sum())
            T = np.where(live, T * (1 - alpha), T)
    return scores
