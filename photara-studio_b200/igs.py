"""ADC-IGS: the reference trainer's default densification rule.

Restates photara's IgsStrategy::refine
(photara/src/splat/densification_igs.cpp:287-520) and the statistics it
reads (accumulate_densification_kernel, photara/src/splat/cuda_ops.cu:
1548-1606, called from trainer.cpp:2441 with the running-max score, the
visibility requirement and the oversize screen threshold). Each refinement:

1. prune masks (cuda_ops.cu:263-302): hard-prune non-finite rows, rows whose
   mean or largest scale leaves 100 x the scene extent; rows below the
   opacity floor are not pruned outright but recycled: at most
   dense_recycle_fraction of the model (hard prunes included), the least
   opaque first; the most opaque non-hard row is always kept; survivors
   beyond the cap drop the least opaque;
2. per-row evidence over the rows kept: candidates (seen at least once),
   oversize priority = accumulated log2 oversize / views, its upper median
   over the positive rows, edge factor 1 + 0.25 min(priority / median, 10);
3. parents, at most `capacity` = cap - survivors (select_igs_parents,
   densification_igs.cpp:226-285): one replacement per pruned row, sampled
   without replacement with weight opacity x edge (Gumbel top-k); then,
   while growth is allowed, the oversized rows (screen > threshold) ranked
   by screen x edge; then a growth sample of round(select_fraction x
   growth candidates) rows with weight score x edge x (2 if oversized),
   growth candidates being rows whose score passes the gradient threshold;
4. every parent splits with the random-axis IGS split (the library's
   split_gaussians kernel, mode igs_random, one N(0,1) per axis); parents'
   and children's Adam state restarts from zero; survivors keep theirs;
5. ADC decay of every row: opacity_decay and scale_decay scaled by the
   remaining training fraction.

Steps 1-3 are `igs_plan` (plain torch, any device); step 4 is `apply_igs`
on this library's kernels. The sampling uses torch's generator instead of the
reference's std::mt19937 stream, so parent choices match the reference in
distribution, not draw for draw.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import torch

from .densify import (KEEP, PRUNE, SPLIT, AdamState, _Ctx, _p, apply_adc_decay, gather_rows,
                      select_rows, split_gaussians)
from . import _lib as L
from .rasterizer import GaussianModel


@dataclass
class IgsOptions:
    """The reference's TrainingOptions defaults that ADC-IGS reads
    (photara/include/splat/options.hpp:158-224, :500-508)."""
    prune_opacity: float = 1.0 / 255.0
    dense_recycle_fraction: float = 0.01
    cap: int = 3_000_000
    densify_gradient_threshold: float = 0.0025
    densify_screen_threshold: float = 0.25
    densify_select_fraction: float = 0.25
    opacity_decay: float = 0.004
    scale_decay: float = 0.0
    start: int = 500
    every: int = 100
    stop: int = 15_000
    grow_stop: int = 0          # 0: half of the iterations (grow_stop_iteration)
    iterations: int = 30_000

    def is_refinement(self, iteration: int) -> bool:
        """is_refinement_iteration (densification.cpp:160-170) for ADC-IGS."""
        return self.start < iteration < self.stop and self.every > 0 and \
            iteration % self.every == 0

    def growth_stop(self) -> int:
        return self.grow_stop if self.grow_stop else max(1, self.iterations // 2)


class IgsStats:
    """DensificationStats (photara/src/splat/ops.hpp:38-52) of this library's
    rows, plus two per-row features of the learned proposal (mean view depth,
    refinement age) that the reference does not keep."""

    NAMES = ("gradient", "count", "max_screen_radius", "priority", "max_geometry_gradient",
             "view_support", "image_error", "depth_acc", "age")

    def __init__(self, n: int, device):
        self.t = {k: torch.zeros(n, device=device) for k in self.NAMES}
        self.t["first_view"] = torch.zeros(n, dtype=torch.int32, device=device)

    def accumulate(self, rendered, refine_weight: torch.Tensor, camera, means: torch.Tensor,
                   view_index: int, opts: IgsOptions) -> None:
        """One view, as the reference trainer accumulates for ADC-IGS
        (trainer.cpp:2441-2450): running-max score, visible rows only, the
        oversize screen threshold, the refine weight as geometry score too."""
        n = rendered.radii.numel()
        a = L.DensifyAccum()
        a.refine_weight = _p(refine_weight)
        a.visibility = _p(rendered.visibility)
        a.radii = _p(rendered.radii)
        for k in ("gradient", "count", "max_screen_radius", "priority", "max_geometry_gradient",
                  "view_support"):
            setattr(a, k, _p(self.t[k]))
        a.geometry_gradient = _p(refine_weight)
        a.first_view = _p(self.t["first_view"])
        a.count_rows = n
        a.inverse_resolution = 1.0 / max(1, min(camera.width, camera.height))
        a.use_maximum = 1
        a.require_visibility = 1
        a.step_score_power = 1.0
        a.oversize_screen_threshold = float(opts.densify_screen_threshold)
        a.view_index = int(view_index)
        with _Ctx(rendered.radii.device.index or 0) as ctx:
            L.check(L.load().gs_accumulate_densification(ctx, a), ctx)
        # view-space depth of the rows this view saw (a feature of the proposal)
        w = [float(v) for v in camera.world_to_camera]  # column-major 4x4
        row = torch.tensor([w[2], w[6], w[10]], device=means.device)
        seen = (rendered.radii > 0) & (rendered.visibility > 0)
        self.t["depth_acc"] += torch.where(seen, means @ row + w[14], 0.0)

    def reset(self, keep_age: bool = True) -> None:
        for k in self.t:
            if k != "age" or not keep_age:
                self.t[k].zero_()

    def remap(self, index: torch.Tensor, n_new: int) -> None:
        """Rows follow the model: `index` selects survivors, new rows start fresh."""
        for k in list(self.t):
            kept = self.t[k].index_select(0, index)
            self.t[k] = torch.cat([kept, torch.zeros(n_new, dtype=kept.dtype,
                                                     device=kept.device)])


def _front(values: torch.Tensor, mask: torch.Tensor, count: int, descending: bool):
    """select_front (densification_igs.cpp:92-123): the `count` rows of `mask`
    first in the requested order of `values` (stable sort, ties by index)."""
    found = min(int(count), int(mask.sum()))
    if found <= 0:
        return values.new_zeros((0,), dtype=torch.int64)
    sentinel = -math.inf if descending else math.inf
    keyed = values.masked_fill(~mask, sentinel)
    order = torch.sort(keyed, descending=descending, stable=True).indices
    return order[:found]


def _gumbel_top(weights: torch.Tensor, requested: int, gen: torch.Generator):
    """weighted_gumbel_sample (densification_igs.cpp:166-224): `requested`
    rows without replacement, P proportional to weight, by the largest
    log(w) - log(-log(u)) over the finite positive weights."""
    if requested <= 0 or weights.numel() == 0:
        return weights.new_zeros((0,), dtype=torch.int64)
    eligible = torch.isfinite(weights) & (weights > 0)
    u = torch.rand(weights.shape, generator=gen, device=weights.device).clamp(1e-7, 1 - 1e-7)
    scores = torch.log(weights.clamp_min(1e-38)) - torch.log(-torch.log(u))
    return _front(scores, eligible, requested, True)


def _upper_median(values: torch.Tensor, positive: torch.Tensor) -> float:
    """positive_upper_median (densification_igs.cpp:147-164): the
    (count / 2 + 1)-th smallest value among the positive rows."""
    cnt = int(positive.sum())
    if cnt == 0:
        return 0.0
    v = torch.sort(values[positive]).values
    return float(v[cnt // 2])


@dataclass
class IgsPlan:
    keep: torch.Tensor              # bool [N]: rows kept
    parents: torch.Tensor           # int64, indices into the KEPT rows, increasing
    pruned: int
    capacity: int
    counts: dict = field(default_factory=dict)
    # per kept row, for the learned proposal and the logs
    candidate: Optional[torch.Tensor] = None
    edge: Optional[torch.Tensor] = None
    growth_mask: Optional[torch.Tensor] = None
    oversized: Optional[torch.Tensor] = None
    replacement_weights: Optional[torch.Tensor] = None
    growth_weights: Optional[torch.Tensor] = None
    oversize_scores: Optional[torch.Tensor] = None
    desired_growth: int = 0


def prune_masks(model: GaussianModel, minimum_opacity: float, maximum_bounds: float,
                center) -> tuple:
    """adc_plus_prune_kernel (cuda_ops.cu:263-302): (keep, hard, opacities)."""
    logits = model.opacity_logits.reshape(-1)
    opacity = torch.sigmoid(logits)
    n = logits.numel()
    bad = ~torch.isfinite(logits)
    bad |= ~torch.isfinite(model.means).all(dim=1) | ~torch.isfinite(model.log_scales).all(dim=1)
    bad |= ~torch.isfinite(model.quaternions).all(dim=1)
    bad |= ~torch.isfinite(model.sh.reshape(n, -1)).all(dim=1)
    max_scale = torch.exp(model.log_scales).amax(dim=1)
    c = torch.tensor([float(v) for v in center], device=model.means.device)
    outside = ((model.means - c).abs() > maximum_bounds).any(dim=1)
    hard = bad | outside | (max_scale > maximum_bounds)
    keep = ~hard & (opacity >= minimum_opacity)
    return keep, hard, opacity


def igs_plan(model: GaussianModel, stats: IgsStats, iteration: int, opts: IgsOptions,
             extent: float, center, gen: torch.Generator,
             growth_override=None, replacement_override=None) -> IgsPlan:
    """Steps 1-3 of IgsStrategy::refine (densification_igs.cpp:287-500).
    replacement_override / growth_override(plan, chosen, count) -> parents
    (kept-row indices, at most `count`, none already chosen) let a learned
    proposal choose the replacement and growth parents in place of the
    weighted samples (it may choose fewer); the prune, recycle, cap and
    oversize rules stay the reference's."""
    n = model.size()
    dev = model.means.device
    keep_m, hard, opacity = prune_masks(model, opts.prune_opacity, 100.0 * extent, center)
    recycled_rows = ~keep_m & ~hard
    keep = ~hard
    hard_count = int(hard.sum())
    recycle_limit = int(math.ceil(n * min(max(opts.dense_recycle_fraction, 0.0), 1.0)))
    budget = recycle_limit - hard_count if recycle_limit > hard_count else 0
    if budget:
        rec = _front(opacity, recycled_rows, budget, False)
        keep[rec] = False
    finite_op = opacity.masked_fill(~torch.isfinite(opacity), -math.inf)
    best = int(torch.argmax(finite_op)) if n else -1
    best_mask = torch.zeros(n, dtype=torch.bool, device=dev)
    if best >= 0:
        best_mask[best] = True
    keep |= best_mask & ~hard
    retained = int(keep.sum())
    if retained > opts.cap:
        removable = keep & ~best_mask
        drop = _front(opacity, removable, retained - opts.cap, False)
        keep[drop] = False
        retained -= int(drop.numel())
    pruned = n - retained
    capacity = opts.cap - retained if opts.cap > retained else 0
    plan = IgsPlan(keep=keep, parents=torch.zeros(0, dtype=torch.int64, device=dev),
                   pruned=pruned, capacity=capacity)
    if capacity == 0:
        return plan
    kidx = torch.nonzero(keep).flatten()
    r_count = stats.t["count"][kidx]
    r_gradient = stats.t["gradient"][kidx]
    r_priority = stats.t["priority"][kidx]
    r_screen = stats.t["max_screen_radius"][kidx]
    r_opacity = opacity[kidx]
    candidate = r_count > 0
    priority = r_priority / r_count.clamp_min(1.0)
    positive = candidate & (priority > 0)
    allow_growth = iteration < opts.growth_stop()
    oversized = candidate & (r_screen > opts.densify_screen_threshold)
    growth_mask = candidate & (r_gradient > opts.densify_gradient_threshold)
    median = max(_upper_median(priority, positive), 1e-9) if int(positive.sum()) else 1.0
    edge = (priority.masked_fill(~(priority > 0), 0.0) / median).clamp_max(10.0) * 0.25 + 1.0
    replacement_w = (r_opacity * edge).masked_fill(~candidate, 0.0)
    growth_w, desired, oversize_s = None, 0, None
    if allow_growth:
        screen_factor = torch.where(oversized, 2.0, 1.0)
        growth_w = (r_gradient * edge * screen_factor).masked_fill(~growth_mask, 0.0)
        desired = int(round(int(growth_mask.sum()) * opts.densify_select_fraction))
        oversize_s = (r_screen * edge).masked_fill(~oversized, 0.0)
    plan.candidate, plan.edge, plan.growth_mask, plan.oversized = (candidate, edge, growth_mask,
                                                                   oversized)
    plan.replacement_weights, plan.growth_weights = replacement_w, growth_w
    plan.oversize_scores, plan.desired_growth = oversize_s, desired
    # select_igs_parents (densification_igs.cpp:226-285)
    chosen = torch.zeros(kidx.numel(), dtype=torch.bool, device=dev)
    if replacement_override is not None:
        repl = replacement_override(plan, chosen, min(pruned, capacity))
    else:
        repl = _gumbel_top(replacement_w, min(pruned, capacity), gen)
    chosen[repl] = True
    remaining = capacity - int(repl.numel())
    n_over = 0
    if remaining and oversize_s is not None:
        eligible = torch.isfinite(oversize_s) & (oversize_s > 0) & ~chosen
        ranked = _front(oversize_s, eligible, remaining, True)
        chosen[ranked] = True
        n_over = int(ranked.numel())
        remaining -= n_over
    n_growth = 0
    if remaining and desired and growth_w is not None:
        want = min(remaining, desired)
        if growth_override is not None:
            grown = growth_override(plan, chosen, want)
        else:
            grown = _gumbel_top(growth_w.masked_fill(chosen, 0.0), want, gen)
        chosen[grown] = True
        n_growth = int(grown.numel())
    plan.parents = torch.nonzero(chosen).flatten()
    plan.counts = {"replacement": int(repl.numel()), "oversized": n_over, "growth": n_growth,
                   "positive": int(positive.sum()), "growth_candidates": int(growth_mask.sum()),
                   "median": median}
    return plan


def apply_igs(model: GaussianModel, adam: AdamState, stats: IgsStats, plan: IgsPlan,
              screen_all: torch.Tensor, iteration: int, opts: IgsOptions,
              gen: torch.Generator) -> tuple[GaussianModel, AdamState, dict]:
    """Step 4 and 5 of IgsStrategy::refine (grow_igs_random_gpu,
    densification_adc_plus.cpp:97-160; apply_adc_decay): survivors first in
    order, then one child per parent; every parent's and child's Adam state
    restarts at zero; the ADC decay scaled by the remaining training fraction.
    Returns (model, adam, info); info["gather"] maps every new row to the
    old row it came from (survivor or parent)."""
    dev = model.means.device
    keep_idx = select_rows(plan.keep.contiguous())
    parents_new = plan.parents.to(torch.int32).contiguous()   # in kept-row numbering
    n_par = int(parents_new.numel())
    fields = ("means", "log_scales", "quaternions", "opacity_logits", "sh")
    parent_old = keep_idx.to(torch.int64)[plan.parents] if n_par else \
        torch.zeros(0, dtype=torch.int64, device=dev)
    gather = torch.cat([keep_idx, parent_old.to(torch.int32)]).contiguous()
    m2 = GaussianModel(*gather_rows(gather, [getattr(model, f) for f in fields]),
                       model.sh_degree)
    s_keys, h_keys = list(adam.structure), list(adam.sh)
    moved = gather_rows(keep_idx, [adam.structure[k] for k in s_keys] +
                        [adam.sh[k] for k in h_keys], rows=int(keep_idx.numel()) + n_par)
    a2 = AdamState()
    a2.structure = dict(zip(s_keys, moved[:len(s_keys)]))
    a2.sh = dict(zip(h_keys, moved[len(s_keys):]))
    if n_par:
        survivors = int(keep_idx.numel())
        children = GaussianModel(m2.means[survivors:], m2.log_scales[survivors:],
                                 m2.quaternions[survivors:], m2.opacity_logits[survivors:],
                                 m2.sh[survivors:], m2.sh_degree)
        samples = torch.randn((n_par, 3), generator=gen, device=dev)
        screens = screen_all[parent_old].contiguous()
        split_gaussians(m2, children, parents_new, "igs_random", random_samples=samples,
                        screen_sizes=screens, minimum_opacity=opts.prune_opacity)
        # the parents' moments restart (keep_parent_adam = false)
        for k in s_keys:
            a2.structure[k][plan.parents] = 0
        for k in h_keys:
            a2.sh[k][plan.parents] = 0
    remaining = 1.0 - iteration / max(1.0, float(opts.iterations))
    apply_adc_decay(m2, opts.opacity_decay * max(remaining, 0.0),
                    opts.scale_decay * max(remaining, 0.0))
    stats.remap(keep_idx.to(torch.int64), n_par)
    info = {"pruned": plan.pruned, "split": n_par, "cloned": 0, "count": m2.size(),
            "gather": gather, **plan.counts}
    return m2, a2, info


def actions_of(plan: IgsPlan, n: int) -> torch.Tensor:
    """Per old row: PRUNE (not kept), SPLIT (parent), KEEP."""
    dev = plan.keep.device
    a = torch.full((n,), KEEP, dtype=torch.int32, device=dev)
    a[~plan.keep] = PRUNE
    if plan.parents.numel():
        kidx = torch.nonzero(plan.keep).flatten()
        a[kidx[plan.parents]] = SPLIT
    return a
