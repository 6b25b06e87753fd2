"""Float64 NumPy restatement of photara's per-view training loss
(cuda_backend::compute_training_loss, photara/src/splat/cuda_ops.cu:2731-2822,
pinhole cameras): loss_kernel (cuda_ops.cu:846-966), the fused L1 + SSIM term
(oracle/ssim_ref.py) and depth_normal_consistency_kernel (cuda_ops.cu:999-1071).

TEST INFRASTRUCTURE ONLY: the checker for the library's training-loss
kernels, used by tests/; never by the product.
"""
from __future__ import annotations

import numpy as np

from . import ssim_ref

ALPHA_MODES = {"validity": -1, "masked": 0, "transparent": 1}


def _f(a):
    return None if a is None else np.asarray(a, np.float64)


def depth_normal_consistency(depth, normal, fx, fy, cx, cy, weight):
    """cuda_ops.cu:999-1071. Returns (loss, grad_depth [H,W], grad_normal [3,H,W])."""
    d = np.asarray(depth, np.float64)
    n = np.asarray(normal, np.float64)
    H, W = d.shape
    gd = np.zeros_like(d)
    gn = np.zeros_like(n)
    norm = weight / (W * H)
    ys, xs = np.mgrid[1:H - 1, 1:W - 1]
    c = d[1:-1, 1:-1]
    top, bottom, left, right = d[:-2, 1:-1], d[2:, 1:-1], d[1:-1, :-2], d[1:-1, 2:]
    ok = (c > 0) & (top > 0) & (bottom > 0) & (left > 0) & (right > 0)

    def ray(px, py):
        return np.stack([(px - cx) / fx, (py - cy) / fy, np.ones_like(px, np.float64)])

    r_t, r_b = ray(xs, ys - 1.0), ray(xs, ys + 1.0)
    r_l, r_r = ray(xs - 1.0, ys), ray(xs + 1.0, ys)
    dy = r_b * bottom - r_t * top
    dx = r_r * right - r_l * left
    cr = np.cross(dy, dx, axis=0)
    l2 = (cr * cr).sum(0)
    ok &= (l2 > 1e-20) & np.isfinite(l2)
    inv = np.where(ok, 1.0 / np.sqrt(np.where(ok, l2, 1.0)), 0.0)
    dn = cr * inv
    raster = n[:, 1:-1, 1:-1]
    loss = float((norm * (1.0 - (raster * dn).sum(0)))[ok].sum())
    gn[:, 1:-1, 1:-1] += np.where(ok, -norm * dn, 0.0)
    gu = -norm * raster
    proj = (dn * gu).sum(0)
    gc = (gu - dn * proj) * inv
    g_dy = np.cross(dx, gc, axis=0)
    g_dx = np.cross(gc, dy, axis=0)
    okf = ok.astype(np.float64)
    gd[2:, 1:-1] += okf * (g_dy * r_b).sum(0)
    gd[:-2, 1:-1] -= okf * (g_dy * r_t).sum(0)
    gd[1:-1, 2:] += okf * (g_dx * r_r).sum(0)
    gd[1:-1, :-2] -= okf * (g_dx * r_l).sum(0)
    return loss, gd, gn


def training_loss(color, target_color, *, alpha=None, median_depth=None, normal=None,
                  target_depth=None, target_normal=None, mask=None, intrinsics=None,
                  photometric_weight=1.0, ssim_weight=0.2, depth_weight=0.0, normal_weight=0.0,
                  depth_normal_weight=0.0, match_alpha_weight=0.25, geometry_epsilon=1e-3,
                  alpha_mode="masked", ai_prior=False, need_geometry_gradients=False):
    """Returns a dict of float64 arrays: color [3,H,W], alpha [H,W], depth and
    normal (or None), terms [4] (rgb, depth, normal, alpha)."""
    color, target_color = _f(color), _f(target_color)
    alpha, median_depth, normal = _f(alpha), _f(median_depth), _f(normal)
    target_depth, target_normal, mask = _f(target_depth), _f(target_normal), _f(mask)
    _, H, W = color.shape
    P = H * W
    mode = ALPHA_MODES[alpha_mode]
    valid = mask if mask is not None else np.ones((H, W))
    inv = 1.0 / P
    fused = W > 10 and H > 10
    photo = 0.0 if fused else photometric_weight
    terms = np.zeros(4)
    diff = color - target_color
    g_color = photo * valid * inv / 3.0 * np.sign(diff)
    if photo != 0.0:
        terms[0] += float((photo * valid * np.abs(diff).sum(0) * inv / 3.0).sum())
    gm = valid if ai_prior else np.ones((H, W))
    g_depth = np.zeros((H, W))
    if depth_weight > 0:
        has = (target_depth > 0) & (median_depth > 0) & (valid > 0)
        scale = np.maximum(target_depth, 1e-4)
        dd = (median_depth - target_depth) / scale
        robust = np.sqrt(dd * dd + geometry_epsilon ** 2)
        g_depth = np.where(has, gm * depth_weight * inv * dd / (robust * scale), 0.0)
        terms[1] += float(np.where(has, gm * depth_weight * robust * inv, 0.0).sum())
    g_normal = np.zeros((3, H, W))
    if normal_weight > 0:
        tl2 = (target_normal ** 2).sum(0)
        has = (tl2 > 0.25) & (valid > 0)
        itl = 1.0 / np.sqrt(np.where(has, tl2, 1.0))
        dot = (normal * target_normal * itl).sum(0)
        terms[2] += float(np.where(has, gm * normal_weight * (1 - dot) * inv, 0.0).sum())
        g_normal = np.where(has, -gm * normal_weight * target_normal * itl * inv, 0.0)
    g_alpha = np.zeros((H, W))
    if mask is not None and mode == 1 and match_alpha_weight > 0:
        # the clamp bounds as the float32 values the kernel uses (1 - 1e-7
        # rounds to 1 - 2^-23 in float32, which the log at saturated pixels sees)
        lo = float(np.float32(1e-7))
        hi = float(np.float32(1.0) - np.float32(1e-7))
        pred = np.clip(alpha, lo, hi)
        inside = (alpha > lo) & (alpha < hi)
        bg = 1 - valid
        g_alpha = np.where(inside, match_alpha_weight * inv * (bg * pred - valid * (1 - pred)) /
                           (pred * (1 - pred)), 0.0)
        terms[3] += float((-match_alpha_weight * inv *
                           (valid * np.log(pred) + bg * np.log(1 - pred))).sum())
    if fused:
        loss, g, _ = ssim_ref.fused_l1_ssim(color, target_color, mask,
                                            min(max(ssim_weight, 0.0), 1.0), photometric_weight)
        g_color = g_color + g
        terms[0] += loss
    if need_geometry_gradients and depth_normal_weight > 0:
        fx, fy, cx, cy = intrinsics
        loss, gd, gn = depth_normal_consistency(median_depth, normal, fx, fy, cx, cy,
                                                depth_normal_weight)
        terms[2] += loss
        g_depth = g_depth + gd
        g_normal = g_normal + gn
    return {"color": g_color, "alpha": g_alpha,
            "depth": g_depth if need_geometry_gradients else None,
            "normal": g_normal if need_geometry_gradients else None, "terms": terms}
