"""NumPy restatement of the densification kernels and the proposal MLP.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of
photara-studio_b200/csrc/densify.cu and csrc/mlp.cu, never by the product.

Follows the same reference behaviour as those kernels:
  statistics  photara/src/splat/cuda_ops.cu:1548-1606 (refine weight summed over
              the views that see a Gaussian, count, max screen radius)
  split       photara/src/splat/cuda_ops.cu:1720-1845 (adc_covariance mode)
and the classic adaptive-density-control rule for the plain decision. The MLP
is evaluated in float64 from the BF16-rounded weights, so the kernel's FP32
accumulation is checked against an exact-arithmetic answer.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 8, 64, 4
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_IN * N_HID
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_HID * N_OUT
N_PARAMS = OFF_B3 + N_OUT
KEEP, SPLIT, CLONE, PRUNE = 0, 1, 2, 3


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[OFF_W1:OFF_B1].reshape(N_IN, N_HID), w[OFF_B1:OFF_W2],
            w[OFF_W2:OFF_B2].reshape(N_HID, N_HID), w[OFF_B2:OFF_W3],
            w[OFF_W3:OFF_B3].reshape(N_HID, N_OUT), w[OFF_B3:N_PARAMS])


def pack(W1, b1, W2, b2, W3, b3):
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, W3.ravel(), b3])


def bf16_round(x):
    """Round-to-nearest-even to bfloat16, returned as float32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def mlp_forward(x, w):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(x, np.float64)
    a1 = x @ W1 + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0)
    return h2 @ W3 + b3, (x, a1, h1, a2, h2)


def mlp_loss_grad(x, labels, row_weights, w, weight_sum):
    """Weighted softmax cross-entropy, sum_r w_r CE_r / weight_sum, and its
    gradient with respect to the packed parameters."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    z, (x, a1, h1, a2, h2) = mlp_forward(x, w)
    wr = np.asarray(row_weights, np.float64) / weight_sum
    zmax = z.max(1, keepdims=True)
    e = np.exp(z - zmax)
    se = e.sum(1, keepdims=True)
    lab = np.asarray(labels, np.int64)
    loss = float((wr * (np.log(se[:, 0]) + zmax[:, 0] - z[np.arange(len(lab)), lab])).sum())
    dz = e / se
    dz[np.arange(len(lab)), lab] -= 1
    dz *= wr[:, None]
    d2 = (dz @ W3.T) * (a2 > 0)
    d1 = (d2 @ W2.T) * (a1 > 0)
    g = pack(x.T @ d1, d1.sum(0), h1.T @ d2, d2.sum(0), h2.T @ dz, dz.sum(0))
    return loss, g


def mlp_adam(master, grad, m, v, lr, b1, b2, c1, c2, eps):
    m[:] = b1 * m + (1 - b1) * grad
    v[:] = b2 * v + (1 - b2) * grad * grad
    master[:] = master - lr * (m / c1) / (np.sqrt(v / c2) + eps)
    return master, bf16_round(master)


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-np.asarray(x, np.float64)))


def accumulate(stats, refine_weight, radii, means, depth_row, inv_resolution,
               densify_weight=None, densify_weight_den=None):
    seen = np.asarray(radii) > 0
    w = np.nan_to_num(np.asarray(refine_weight, np.float64), nan=0.0, posinf=0.0, neginf=0.0)
    stats["grad_acc"][seen] += np.maximum(w[seen], 0)
    stats["count"][seen] += 1
    stats["max_screen"][seen] = np.maximum(stats["max_screen"][seen],
                                           np.asarray(radii)[seen] * inv_resolution)
    r = np.asarray(depth_row, np.float64)
    m = np.asarray(means, np.float64)
    stats["depth_acc"][seen] += m[seen] @ r[:3] + r[3]
    if densify_weight is not None:
        stats["err_num"][seen] += np.asarray(densify_weight)[seen]
        stats["err_den"][seen] += np.asarray(densify_weight_den)[seen]
    return stats


def features(means, log_scales, logits, sh_dc, stats, center, extent, norm=None):
    cnt = stats["count"].astype(np.float64)
    grad = stats["grad_acc"] / np.maximum(cnt, 1)
    ls = np.asarray(log_scales, np.float64)
    d = np.asarray(means, np.float64) - np.asarray(center, np.float64)
    dist = np.sqrt((d * d).sum(1))
    depth = np.where(cnt > 0, stats["depth_acc"] / np.maximum(cnt, 1), dist)
    f = np.stack([np.log(grad + 1e-8), ls.max(1), ls.min(1),
                  sigmoid(np.asarray(logits).reshape(-1)), np.log1p(cnt),
                  np.sqrt((np.asarray(sh_dc, np.float64) ** 2).sum(1)),
                  np.log(np.maximum(depth, 0) / extent + 1e-6), stats["age"]], 1)
    if norm is not None:
        f = (f - norm[:8]) * norm[8:]
    return f


def adc_decide(log_scales, logits, stats, p):
    """p: dict grad_threshold, percent_dense, extent, prune_opacity,
    prune_world_scale, prune_screen, densify."""
    op = sigmoid(np.asarray(logits).reshape(-1))
    max_scale = np.exp(np.asarray(log_scales, np.float64).max(1))
    prune = ~(op >= p["prune_opacity"]) | (max_scale > p["prune_world_scale"] * p["extent"])
    if p["prune_screen"] > 0:
        prune |= stats["max_screen"] > p["prune_screen"]
    act = np.zeros(len(op), np.int32)
    if p["densify"]:
        grad = stats["grad_acc"] / np.maximum(stats["count"], 1)
        dens = grad >= p["grad_threshold"]
        act[dens] = np.where(max_scale[dens] > p["percent_dense"] * p["extent"], SPLIT, CLONE)
    act[prune] = PRUNE
    return act


def proposal_policy(logits, fallback, count, min_confidence):
    z = np.asarray(logits, np.float64)
    best = z.argmax(1)
    conf = 1.0 / np.exp(z - z.max(1, keepdims=True)).sum(1)
    act = np.where(conf >= min_confidence, best, fallback)
    unseen_dens = ((act == SPLIT) | (act == CLONE)) & ~(count > 0)
    act = np.where(unseen_dens, fallback, act)
    act = np.where(fallback == PRUNE, PRUNE, act)
    return act.astype(np.int32)


def quat_rows(q):
    """Rows of the rotation matrix of a scalar-first quaternion (world -> local)."""
    w, x, y, z = np.asarray(q, np.float64) / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)],
                     [2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x)],
                     [2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)]])


def split(means, log_scales, quats, logits, parents, child0):
    """Covariance-preserving split (in place on copies; returns them)."""
    means, log_scales, logits = (np.array(a, np.float64) for a in (means, log_scales, logits))
    logits = logits.reshape(-1)
    k = 1 / np.sqrt(2)
    for c, p in enumerate(parents):
        c += child0
        ls = log_scales[p].copy()
        major = int(np.argmax(ls))
        local = np.zeros(3)
        local[major] = np.sqrt(1 - k * k) * np.exp(ls[major])
        off = quat_rows(quats[p]).T @ local
        centre = means[p].copy()
        means[p], means[c] = centre - off, centre + off
        log_scales[p, major] = log_scales[c, major] = ls[major] + np.log(k)
        op = sigmoid(logits[p])
        rev = np.clip(1 - (1 - op) ** k, 1e-6, 1 - 1e-6)
        logits[p] = logits[c] = np.log(rev / (1 - rev))
    return means, log_scales, logits


def covariance(log_scales, q):
    R = quat_rows(q)
    S = np.diag(np.exp(2 * np.asarray(log_scales, np.float64)))
    return R.T @ S @ R
