"""NumPy restatement of the deterministic part of the reference's ADC-IGS
refinement, for the CPU tests of photara-studio_b200/igs.py.

TEST INFRASTRUCTURE ONLY (the checker): follows
photara/src/splat/cuda_ops.cu:263-302 (adc_plus_prune_kernel: hard prune and
opacity keep masks) and photara/src/splat/densification_igs.cpp:333-470
(low-opacity recycling, the most-opaque rescue, the cap, candidates, oversize
priority, its upper median, edge factors, the replacement, growth and oversize
weights and the desired growth count), row by row with Python loops and
numpy sorts where the reference sorts. The Gumbel top-k draws are not
restated (they are random); the tests check their invariants.
"""
from __future__ import annotations

import math

import numpy as np


def _sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x.astype(np.float64)))


def igs_reference(means, log_scales, quats, logits, sh, count, gradient, priority, screen,
                  iteration, extent, center, prune_opacity=1 / 255, recycle_fraction=0.01,
                  cap=3_000_000, grad_threshold=0.0025, screen_threshold=0.25,
                  select_fraction=0.25, grow_stop=15_000):
    n = means.shape[0]
    opacity = _sigmoid(logits.reshape(-1)).astype(np.float32)
    hard = np.zeros(n, bool)
    keep_m = np.zeros(n, bool)
    bound = 100.0 * extent
    for i in range(n):
        bad = not np.isfinite(logits.reshape(-1)[i])
        bad |= not (np.isfinite(means[i]).all() and np.isfinite(log_scales[i]).all())
        bad |= not np.isfinite(quats[i]).all()
        bad |= not np.isfinite(sh[i]).all()
        out = (np.abs(means[i] - np.asarray(center)) > bound).any()
        h = bad or out or np.exp(log_scales[i]).max() > bound
        hard[i] = h
        keep_m[i] = (not h) and opacity[i] >= prune_opacity
    recycled_rows = ~keep_m & ~hard
    keep = ~hard
    hard_count = int(hard.sum())
    limit = int(math.ceil(n * min(max(recycle_fraction, 0.0), 1.0)))
    budget = limit - hard_count if limit > hard_count else 0
    if budget:
        rows = sorted((float(opacity[i]), i) for i in range(n) if recycled_rows[i])
        for _, i in rows[:budget]:
            keep[i] = False
    fin = np.where(np.isfinite(opacity), opacity, -np.inf)
    best = int(np.argmax(fin))
    if not hard[best]:
        keep[best] = True
    retained = int(keep.sum())
    if retained > cap:
        rows = sorted((float(opacity[i]), i) for i in range(n) if keep[i] and i != best)
        for _, i in rows[:retained - cap]:
            keep[i] = False
        retained = int(keep.sum())
    pruned = n - retained
    capacity = cap - retained if cap > retained else 0
    out = {"keep": keep, "pruned": pruned, "capacity": capacity}
    if capacity == 0:
        return out
    k = np.nonzero(keep)[0]
    c, g, p, s, o = count[k], gradient[k], priority[k], screen[k], opacity[k]
    candidate = c > 0
    prio = (p / np.maximum(c, 1.0)).astype(np.float32)
    positive = candidate & (prio > 0)
    if positive.sum():
        vals = np.sort(prio[positive])
        median = max(float(vals[positive.sum() // 2]), 1e-9)
    else:
        median = 1.0
    edge = (np.minimum(np.where(prio > 0, prio, 0.0) / np.float32(median), 10.0) * 0.25 +
            1.0).astype(np.float32)
    oversized = candidate & (s > screen_threshold)
    growth_mask = candidate & (g > grad_threshold)
    out.update(candidate=candidate, priority=prio, median=median, edge=edge,
               oversized=oversized, growth_mask=growth_mask,
               replacement_weights=np.where(candidate, o * edge, 0.0).astype(np.float32))
    if iteration < grow_stop:
        factor = np.where(oversized, 2.0, 1.0)
        out["growth_weights"] = np.where(growth_mask, g * edge * factor, 0.0).astype(np.float32)
        out["oversize_scores"] = np.where(oversized, s * edge, 0.0).astype(np.float32)
        out["desired_growth"] = int(round(int(growth_mask.sum()) * select_fraction))
    return out
