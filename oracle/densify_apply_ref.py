"""Float64 NumPy restatement of photara's densification apply operators:
the four split modes of split_gaussians_kernel (photara/src/splat/
cuda_ops.cu:1720-1845, clamps of cuda_backend::split_gaussians at
:3105-3122), the ADC decay (adc_decay_kernel :1847-1861, host clamps
:3388-3400), and the row selection of select_training_rows_gpu
(densification_adc_plus.cpp:68-77).

TEST INFRASTRUCTURE ONLY: the checker for the library's densification
apply kernels, used by tests/; never by the product.
"""
from __future__ import annotations

import numpy as np

MODES = ("adc_covariance", "dense_tangent", "igs_random", "long_axis")


def _sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def _logit(p):
    return np.log(p / (1.0 - p))


def rotate(q, v):
    """Rotate v [n,3] by the normalised quaternions q [n,4] (w, x, y, z)."""
    q = q / np.sqrt(np.maximum((q * q).sum(1, keepdims=True), 1e-20))
    w, u = q[:, :1], q[:, 1:]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def split(parent, child, parents, mode, random_samples=None, screen_sizes=None,
          minimum_opacity=1e-6, split_at_screen_size=0.0, split_opacity_k=0.5):
    """Returns updated copies (dicts of float64 arrays: means [n,3], log_scales
    [n,3], opacity_logits [n], quaternions [n,4]) of parent and child."""
    P = {k: np.array(v, np.float64) for k, v in parent.items()}
    Cc = {k: np.array(v, np.float64) for k, v in child.items()}
    idx = np.asarray(parents, np.int64)
    m = len(idx)
    min_op = min(max(minimum_opacity, 1e-8), 0.49)
    at_screen = max(split_at_screen_size, 0.0)
    kk = min(max(split_opacity_k, 1e-4), 1 - 1e-4)
    ls = P["log_scales"][idx]
    local = np.zeros((m, 3))
    delta = np.zeros((m, 3))
    rows = np.arange(m)
    if mode == "dense_tangent":
        rs = np.asarray(random_samples, np.float64)
        local[:, 0] = np.exp(ls[:, 0]) * rs[:, 0] * 0.5
        local[:, 1] = np.exp(ls[:, 1]) * rs[:, 1] * 0.5
        delta[:, :2] = np.log(0.7071067811865475)
    elif mode == "adc_covariance":
        major = np.argmax(np.exp(ls) ** 2, axis=1)  # first of equal maxima
        k_std = 1.0 / np.sqrt(2.0)
        if screen_sizes is not None and at_screen > 0:
            screen = np.maximum(np.asarray(screen_sizes, np.float64), 1e-6)
            kmax = np.minimum(k_std, at_screen / screen)
        else:
            kmax = np.full(m, k_std)
        local[rows, major] = np.sqrt(np.maximum(1 - kmax ** 2, 0)) * np.exp(ls[rows, major])
        delta[rows, major] = np.log(np.maximum(kmax, 1e-12))
    elif mode == "igs_random":
        largest = np.argmax(ls, axis=1)
        rs = np.asarray(random_samples, np.float64)
        local = np.exp(ls) * rs[:, :1]
        delta[rows, largest] = np.log(0.5)
    elif mode == "long_axis":
        largest = np.argmax(ls, axis=1)
        local[rows, largest] = 0.5 * np.exp(ls[rows, largest])
        delta[:] = np.log(0.85)
        delta[rows, largest] = np.log(0.5)
    else:
        raise ValueError(mode)
    off = rotate(P["quaternions"][idx], local)
    center = P["means"][idx]
    P["means"][idx] = center - off
    Cc["means"][:m] = center + off
    P["log_scales"][idx] += delta
    Cc["log_scales"][:m] += delta
    logit_p = P["opacity_logits"][idx]
    # clamp bounds as the float32 values the kernel compares with (1 - 1e-6 is
    # 1 - 1.013e-6 in float32, which the logit of a clamped opacity sees)
    f32 = lambda x: float(np.float32(x))
    if mode == "long_axis":
        lo, hi = f32(1e-6), float(np.float32(1.0) - np.float32(1e-6))
        den = 1.0 + np.exp(-logit_p) - kk
        mapped = np.where(den > 1e-6, np.clip(kk / np.where(den > 1e-6, den, 1.0), lo, hi), hi)
        new = _logit(mapped)
    else:
        lo, hi = f32(min_op), float(np.float32(1.0) - np.float32(min_op))
        a = _sigmoid(logit_p)
        power = 1.0 / np.sqrt(2.0) if mode == "adc_covariance" else 0.5
        rev = np.clip(1.0 - np.maximum(1.0 - a, 0.0) ** power, lo, hi)
        new = _logit(rev)
    P["opacity_logits"][idx] = new
    Cc["opacity_logits"][:m] = new
    return P, Cc


def adc_decay(log_scales, opacity_logits, opacity_decay, scale_decay):
    ls = np.array(log_scales, np.float64)
    lo = np.array(opacity_logits, np.float64)
    op = np.clip(_sigmoid(lo) - max(opacity_decay, 0.0), 1e-12, 1 - 1e-12)
    return ls + np.log(max(1.0 - scale_decay, 1e-6)), _logit(op)


def select_rows(keep):
    return np.flatnonzero(np.asarray(keep) != 0).astype(np.int32)
