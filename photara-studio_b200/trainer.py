"""Training loop with densification (the reference's ADC-IGS rule, the
learned proposal MLP over it, or the classic ADC rule).

A compact restatement of the reference trainer's loop skeleton
(photara/src/splat/trainer.cpp:1818 loop, :2024 forward, :2379 backward with
fused Adam, :2441 densification statistics, :2571 refinement) on this
library's kernels, for the densification experiment: a synthetic ground-truth
scene is rendered to training and held-out views, a model is initialised from
noisy ground-truth points and trained with L1; densification runs every
`every` iterations in [start, stop]; held-out PSNR = -10 log10(MSE)
(trainer.cpp:2957-2962) is logged against training time.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from .densify import (CLONE, KEEP, PRUNE, SPLIT, AdamState, DensifyConfig, DensifyStats,
                      ProposalMLP, adc_decide, apply_actions, features, reset_opacity)
from . import igs as IGS
from .rasterizer import (Camera, GaussianModel, RasterizeOptions, Rasterizer, SHAdamUpdate,
                         StructureAdamUpdate, look_at_camera)


@dataclass
class SceneSet:
    gt: GaussianModel
    train: list
    test: list
    train_images: list
    test_images: list
    center: tuple
    extent: float


def make_ring_scene(n_gt=500_000, half=3.0, n_train=24, n_test=8, width=1280, height=720,
                    radius=4.0, fx=800.0, seed=0, device="cuda") -> SceneSet:
    """Ground truth: n_gt Gaussians (log-scales N(-3.5,0.5), quaternions
    normalised N(0,1)^4, opacity sigmoid(N(0,1)), SH degree 3 with DC N(0,0.3)
    and rest N(0,0.05)), means uniform in [-half, half]^3; views on a ring of
    `radius` looking at the origin, every 4th one held out."""
    rng = np.random.default_rng(seed)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device)
    means = rng.uniform(-half, half, size=(n_gt, 3))
    ls = rng.normal(-3.5, 0.5, size=(n_gt, 3))
    q = rng.normal(size=(n_gt, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    lo = rng.normal(size=(n_gt, 1))
    sh = np.empty((n_gt, 16, 3))
    sh[:, 0] = rng.normal(0, 0.3, size=(n_gt, 3))
    sh[:, 1:] = rng.normal(0, 0.05, size=(n_gt, 15, 3))
    gt = GaussianModel(t(means), t(ls), t(q), t(lo), t(sh), 3)
    views = n_train + n_test
    cams = []
    for k in range(views):
        a = 2 * math.pi * k / views
        eye = (radius * math.cos(a), 0.6, radius * math.sin(a))
        cams.append(look_at_camera(eye, (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), width, height, fx))
    test_idx = set(range(0, views, views // n_test))
    train = [c for k, c in enumerate(cams) if k not in test_idx]
    test = [c for k, c in enumerate(cams) if k in test_idx]
    rast = Rasterizer()
    opts = RasterizeOptions(active_sh_degree=3, record_backward_state=False)
    render = lambda c: rast.forward(gt, c, opts).color.clone()
    return SceneSet(gt, train, test, [render(c) for c in train], [render(c) for c in test],
                    (0.0, 0.0, 0.0), radius * 1.1)


def init_from_points(scene: SceneSet, n=100_000, noise=0.05, seed=1) -> GaussianModel:
    """n points = ground-truth means + N(0, noise); DC colour from those points
    (a coloured point cloud), isotropic scales, opacity 0.1."""
    g = torch.Generator(device=scene.gt.means.device).manual_seed(seed)
    dev = scene.gt.means.device
    idx = torch.randperm(scene.gt.size(), generator=g, device=dev)[:n]
    means = scene.gt.means[idx] + noise * torch.randn((n, 3), generator=g, device=dev)
    log_scales = torch.full((n, 3), math.log(0.04), device=dev)
    quats = torch.zeros((n, 4), device=dev)
    quats[:, 0] = 1
    logits = torch.full((n, 1), math.log(0.1 / 0.9), device=dev)
    sh = torch.zeros((n, 16, 3), device=dev)
    sh[:, 0] = scene.gt.sh[idx, 0]
    return GaussianModel(means.contiguous(), log_scales, quats, logits, sh.contiguous(), 3)


def igs_features(model: GaussianModel, stats: "IGS.IgsStats", center, extent: float):
    """The proposal network's eight inputs from the IGS statistics: log running
    max of the refine weight, max / min log-scale, opacity, log(1 + views),
    SH DC norm, log(mean view depth / extent) (distance to the centre for an
    unseen row), refinement age."""
    t = stats.t
    cnt = t["count"]
    dev = model.means.device
    c = torch.tensor([float(v) for v in center], device=dev)
    dist = (model.means - c).norm(dim=1)
    depth = torch.where(cnt > 0, t["depth_acc"] / cnt.clamp_min(1.0), dist)
    ls = model.log_scales
    f = torch.stack([torch.log(t["gradient"] + 1e-8), ls.amax(dim=1), ls.amin(dim=1),
                     torch.sigmoid(model.opacity_logits.reshape(-1)), torch.log1p(cnt),
                     model.sh[:, 0].norm(dim=1), torch.log(depth.clamp_min(0.0) / extent + 1e-6),
                     t["age"]], dim=1)
    return f.contiguous()


@dataclass
class TrainConfig:
    iterations: int = 30_000
    policy: str = "plain"            # plain (ADC-IGS) | learned | adc (classic rule) | none
    densify: DensifyConfig = field(default_factory=DensifyConfig)
    means_lr: float = 1.6e-4         # times the scene extent, decayed to 1/100
    scales_lr: float = 5e-3
    quats_lr: float = 1e-3
    opacity_lr: float = 5e-2
    sh0_lr: float = 2.5e-3
    sh_rest_lr: float = 1.25e-4
    sh_up_every: int = 1_000
    eval_every: int = 500
    seed: int = 0
    sh_reg: float = 0.001            # mean-square prior on non-DC SH (reference default)
    explore: float = 0.0             # random densifications per refinement, x the plain count
    explore_min: int = 500           # ... and at least this many (logging runs)
    log_decisions: bool = False      # log decisions with held-out outcomes (MLP training rows)
    min_confidence: float = 0.5
    budget_factor: float = 1.0       # learned densifications per refinement, x the plain count
    igs: "IGS.IgsOptions" = field(default_factory=lambda: IGS.IgsOptions())


def heldout_error(model: GaussianModel, scene: SceneSet, sh_degree: int):
    """Per-Gaussian held-out error: over the held-out views, the mean absolute
    colour error of the pixels a Gaussian reaches, weighted by its
    contribution alpha * T. Returns (num, den) with error = num / den."""
    n = model.size()
    dev = model.means.device
    num = torch.zeros(n, device=dev)
    den = torch.zeros(n, device=dev)
    rast = Rasterizer()
    opts = RasterizeOptions(active_sh_degree=sh_degree)
    for c, img in zip(scene.test, scene.test_images):
        r = rast.forward(model, c, opts)
        err = (r.color - img).abs().mean(0).contiguous()
        rast.attribute_error(model, r, err, num, den)
        del r
    return num, den


def psnr(model, cams, images, sh_degree) -> float:
    rast = Rasterizer()
    opts = RasterizeOptions(active_sh_degree=sh_degree, record_backward_state=False)
    mse = 0.0
    for c, img in zip(cams, images):
        r = rast.forward(model, c, opts)
        mse += float(((r.color - img) ** 2).mean())
    mse /= len(cams)
    return -10.0 * math.log10(max(mse, 1e-20))


def train(scene: SceneSet, cfg: TrainConfig, model: Optional[GaussianModel] = None,
          mlp: Optional[ProposalMLP] = None) -> dict:
    if cfg.policy in ("plain", "learned"):
        return train_igs(scene, cfg, model, mlp)
    return train_adc(scene, cfg, model, mlp)


def _learned_parents(mlp: ProposalMLP, feats_raw: torch.Tensor, min_confidence: float):
    """Parent choice for igs_plan's replacement and growth draws: the
    network's split + clone probability ranks the candidate rows not chosen
    yet (the rows the statistics saw); at most `want` of the rows whose
    probability reaches min_confidence split (the network may decline)."""
    p = torch.softmax(mlp.logits(mlp.normalise(feats_raw)), dim=1)
    score_all = p[:, SPLIT] + p[:, CLONE]

    def pick(plan, chosen, want):
        score = score_all[torch.nonzero(plan.keep).flatten()]
        return IGS._front(score, plan.candidate & ~chosen & (score >= min_confidence), want,
                          True)
    return pick


def train_igs(scene: SceneSet, cfg: TrainConfig, model: Optional[GaussianModel] = None,
              mlp: Optional[ProposalMLP] = None) -> dict:
    """Training with the reference's ADC-IGS refinement (policy "plain"), or
    with the proposal network choosing the replacement and growth parents
    (policy "learned", at most IGS's counts, declining where it is not
    confident; the prune, recycle, cap and oversize rules stay IGS's)."""
    dev = scene.gt.means.device
    model = model or init_from_points(scene, seed=cfg.seed + 1)
    adam = AdamState.zeros(model)
    iopt = IGS.IgsOptions(**{**vars(cfg.igs), "iterations": cfg.iterations})
    stats = IGS.IgsStats(model.size(), dev)
    rast = Rasterizer()
    lib = L.load()
    rng = np.random.default_rng(cfg.seed)
    gen = torch.Generator(device=dev).manual_seed(cfg.seed)
    H, W = scene.train_images[0].shape[1:]
    grad_color = torch.empty((3, H, W), device=dev)
    loss_buf = torch.zeros(1, device=dev)
    history, samples, outcomes, refinements = [], [], [], []
    pending = None
    t_start = time.perf_counter()
    eval_time = 0.0
    for it in range(1, cfg.iterations + 1):
        sh_degree = min(3, (it - 1) // cfg.sh_up_every)
        k = int(rng.integers(len(scene.train)))
        cam, target = scene.train[k], scene.train_images[k]
        opts = RasterizeOptions(active_sh_degree=sh_degree)
        r = rast.forward(model, cam, opts)
        loss_buf.zero_()
        live = r.context
        L.check(lib.gs_l1_loss(live.ctx.ptr, r.color.data_ptr(), target.data_ptr(), W * H, 1.0,
                               grad_color.data_ptr(), loss_buf.data_ptr()), live.ctx.ptr)
        c1, c2 = 1 - 0.9 ** it, 1 - 0.999 ** it
        frac = it / cfg.iterations
        mlr = cfg.means_lr * scene.extent * (0.01 ** frac)
        sa = StructureAdamUpdate(**adam.structure, means_lr=mlr, scales_lr=cfg.scales_lr,
                                 quaternions_lr=cfg.quats_lr, opacities_lr=cfg.opacity_lr,
                                 correction1=c1, correction2=c2)
        sha = SHAdamUpdate(**adam.sh, lr=cfg.sh0_lr, rest_lr=cfg.sh_rest_lr, correction1=c1,
                           correction2=c2, regularization_weight=cfg.sh_reg)
        grads = rast.backward(model, r, grad_color, None, sh_adam=sha, structure_adam=sa)
        if it <= iopt.stop:
            stats.accumulate(r, grads.refine_weight, cam, model.means, k, iopt)
        del r, live
        if iopt.is_refinement(it):
            held = heldout_error(model, scene, sh_degree) if cfg.log_decisions else None
            if pending is not None:
                closed = _close_log(pending, *held)
                samples.append(labels_from_logs([closed], seed=it))
                outcomes.append(densify_outcomes(closed))
                pending = None
            feats_raw = None
            if cfg.policy == "learned" or cfg.log_decisions:
                feats_raw = igs_features(model, stats, scene.center, scene.extent)
            override = None
            if cfg.policy == "learned" and mlp is not None:
                override = _learned_parents(mlp, feats_raw, cfg.min_confidence)
            plan = IGS.igs_plan(model, stats, it, iopt, scene.extent, scene.center, gen,
                                growth_override=override, replacement_override=override)
            plain_parents = plan.parents.clone()
            if cfg.explore > 0 and plan.capacity > 0 and plan.candidate is not None:
                k_x = max(cfg.explore_min, int(cfg.explore * plain_parents.numel()))
                room = plan.capacity - int(plan.parents.numel())
                chosen = torch.zeros_like(plan.candidate)
                chosen[plan.parents] = True
                pool = torch.nonzero(plan.candidate & ~chosen).flatten()
                k_x = min(k_x, room, int(pool.numel()))
                if k_x > 0:
                    extra = pool[torch.randperm(pool.numel(), generator=gen, device=dev)[:k_x]]
                    plan.parents = torch.sort(torch.cat([plan.parents, extra])).values
            old_n = model.size()
            action = IGS.actions_of(plan, old_n)
            plain_dens = torch.zeros(old_n, dtype=torch.bool, device=dev)
            if plain_parents.numel():
                plain_dens[torch.nonzero(plan.keep).flatten()[plain_parents]] = True
            e_before = held[0] / held[1].clamp_min(1e-8) if cfg.log_decisions else None
            model, adam, info = IGS.apply_igs(model, adam, stats, plan,
                                              stats.t["max_screen_radius"], it, iopt, gen)
            refinements.append({"iteration": it, "pruned": info["pruned"],
                                "split": info["split"], "gaussians": info["count"],
                                **{k2: info[k2] for k2 in ("replacement", "oversized", "growth")
                                   if k2 in info}})
            if cfg.log_decisions:
                pending = {"feats": feats_raw, "action": action, "old_n": old_n,
                           "gather": info["gather"], "e_before": e_before,
                           "plain_dens": plain_dens}
            stats.reset()
            stats.t["age"] += 1
        if it % cfg.eval_every == 0 or it == cfg.iterations:
            torch.cuda.synchronize()
            e0 = time.perf_counter()
            p = psnr(model, scene.test, scene.test_images, sh_degree)
            eval_time += time.perf_counter() - e0
            train_time = (time.perf_counter() - t_start) - eval_time
            history.append({"iteration": it, "seconds": train_time, "psnr": p,
                            "gaussians": model.size()})
    return {"history": history, "model": model, "samples": samples, "outcomes": outcomes,
            "refinements": refinements}


def train_adc(scene: SceneSet, cfg: TrainConfig, model: Optional[GaussianModel] = None,
              mlp: Optional[ProposalMLP] = None) -> dict:
    """Training with the classic 3DGS clone / split / prune rule (policy
    "adc"; the learned policy over it is "adc_learned")."""
    dev = scene.gt.means.device
    model = model or init_from_points(scene, seed=cfg.seed + 1)
    adam = AdamState.zeros(model)
    stats = DensifyStats(model.size(), dev)
    rast = Rasterizer()
    lib = L.load()
    rng = np.random.default_rng(cfg.seed)
    H, W = scene.train_images[0].shape[1:]
    grad_color = torch.empty((3, H, W), device=dev)
    loss_buf = torch.zeros(1, device=dev)
    history, samples, outcomes, refinements = [], [], [], []
    pending = None  # decision log waiting for its outcome window
    train_time = 0.0
    t_start = time.perf_counter()
    eval_time = 0.0
    dcfg = cfg.densify
    for it in range(1, cfg.iterations + 1):
        sh_degree = min(3, (it - 1) // cfg.sh_up_every)
        k = int(rng.integers(len(scene.train)))
        cam, target = scene.train[k], scene.train_images[k]
        opts = RasterizeOptions(active_sh_degree=sh_degree)
        r = rast.forward(model, cam, opts)
        loss_buf.zero_()
        live = r.context
        L.check(lib.gs_l1_loss(live.ctx.ptr, r.color.data_ptr(), target.data_ptr(), W * H, 1.0,
                               grad_color.data_ptr(), loss_buf.data_ptr()), live.ctx.ptr)
        t = it
        c1, c2 = 1 - 0.9 ** t, 1 - 0.999 ** t
        frac = it / cfg.iterations
        mlr = cfg.means_lr * scene.extent * (0.01 ** frac)
        sa = StructureAdamUpdate(**adam.structure, means_lr=mlr, scales_lr=cfg.scales_lr,
                                 quaternions_lr=cfg.quats_lr, opacities_lr=cfg.opacity_lr,
                                 correction1=c1, correction2=c2)
        sha = SHAdamUpdate(**adam.sh, lr=cfg.sh0_lr, rest_lr=cfg.sh_rest_lr, correction1=c1,
                           correction2=c2, regularization_weight=cfg.sh_reg)
        grads = rast.backward(model, r, grad_color, None, sh_adam=sha, structure_adam=sa)
        in_window = dcfg.start - dcfg.every <= it <= dcfg.stop + dcfg.every
        if cfg.policy != "none" and in_window:
            stats.accumulate(r, grads, cam, model.means)
        del r, live
        if cfg.policy != "none" and dcfg.start <= it <= dcfg.stop and it % dcfg.every == 0:
            held = heldout_error(model, scene, sh_degree) if cfg.log_decisions else None
            if pending is not None:
                closed = _close_log(pending, *held)
                samples.append(labels_from_logs([closed], seed=it))
                outcomes.append(densify_outcomes(closed))
                pending = None
            screen_rule = dcfg.opacity_reset_every <= 0 or it > dcfg.opacity_reset_every
            action = adc_decide(model, stats, dcfg, scene.extent, prune_screen=screen_rule)
            feats_raw = None
            if cfg.policy == "adc_learned" or cfg.log_decisions:
                feats_raw = features(model, stats, scene.center, scene.extent)
            plain_dens = (action == SPLIT) | (action == CLONE)
            plain_count = int(plain_dens.sum())
            if cfg.policy == "adc_learned" and mlp is not None:
                action = mlp.propose_budget(feats_raw, action, stats,
                                            int(round(cfg.budget_factor * plain_count)),
                                            cfg.min_confidence)
            if cfg.explore > 0:
                k = max(cfg.explore_min, int(cfg.explore * plain_count))
                action = _explore(action, stats, model, dcfg, scene.extent, k, rng)
            old_n = model.size()
            e_before = held[0] / held[1].clamp_min(1e-8) if cfg.log_decisions else None
            model, adam, info = apply_actions(model, adam, stats, action, dcfg.cap)
            refinements.append({"iteration": it, "pruned": info["pruned"],
                                "split": info["split"], "cloned": info["cloned"],
                                "gaussians": info["count"]})
            if cfg.log_decisions:
                pending = {"feats": feats_raw, "action": action, "old_n": old_n,
                           "gather": info["gather"], "e_before": e_before,
                           "plain_dens": plain_dens}
            stats.reset()
            stats.t["age"] += 1
        if it % cfg.eval_every == 0 or it == cfg.iterations:
            torch.cuda.synchronize()
            e0 = time.perf_counter()
            p = psnr(model, scene.test, scene.test_images, sh_degree)
            eval_time += time.perf_counter() - e0
            train_time = (time.perf_counter() - t_start) - eval_time
            history.append({"iteration": it, "seconds": train_time, "psnr": p,
                            "gaussians": model.size()})
        if cfg.policy != "none" and dcfg.opacity_reset_every and it % dcfg.opacity_reset_every == 0 \
                and it < dcfg.stop:
            reset_opacity(model)
            adam.structure["opacity_first"].zero_()
            adam.structure["opacity_second"].zero_()
    return {"history": history, "model": model, "samples": samples, "outcomes": outcomes,
            "refinements": refinements}


def _close_log(pending: dict, num_rows: torch.Tensor, den_rows: torch.Tensor) -> dict:
    """Outcome of a logged decision: the held-out error seen by the rows
    derived from each old Gaussian one window later, beside its error at the
    decision."""
    gather = pending["gather"].to(torch.int64)
    n_old = pending["old_n"]
    num = torch.zeros(n_old, device=gather.device).index_add_(0, gather, num_rows[:gather.numel()])
    den = torch.zeros(n_old, device=gather.device).index_add_(0, gather, den_rows[:gather.numel()])
    e_after = num / den.clamp_min(1e-8)
    seen = den > 0
    e_before = pending["e_before"][:n_old]
    return {"feats": pending["feats"], "action": pending["action"], "e_before": e_before,
            "e_after": e_after, "seen_after": seen, "plain_dens": pending["plain_dens"]}


def _explore(action, stats, model, dcfg, extent, k, rng):
    """Random densify decisions for `k` seen, kept Gaussians so the logs hold
    outcomes of actions the plain rule would not take (split or clone by the
    plain size rule)."""
    seen = torch.nonzero((stats.t["count"] > 0) & (action == KEEP)).flatten()
    if seen.numel() == 0 or k <= 0:
        return action
    g = torch.Generator(device=action.device).manual_seed(int(rng.integers(1 << 31)))
    pick = seen[torch.randperm(seen.numel(), generator=g, device=action.device)[:k]]
    big = torch.exp(model.log_scales[pick].max(dim=1).values) > dcfg.percent_dense * extent
    out = action.clone()
    out[pick] = torch.where(big, SPLIT, CLONE).to(out.dtype)
    return out


def _adjusted_gain(log: dict):
    """Relative drop of the held-out error each logged Gaussian (or the rows
    derived from it) saw over the next window, minus the median drop of the
    kept Gaussians (the drift every row sees); and the mask of densified rows
    with a measured outcome."""
    a = log["action"].to(torch.int64)
    eb, ea, seen = log["e_before"], log["e_after"], log["seen_after"]
    gain = (eb - ea) / eb.clamp_min(1e-8)
    kept_seen = (a == KEEP) & seen & (eb > 0)
    if int(kept_seen.sum()) > 0:
        gain = gain - gain[kept_seen].median()
    dens = ((a == SPLIT) | (a == CLONE)) & seen & (eb > 0)
    return gain, dens


def densify_outcomes(log: dict):
    """(features, adjusted gain, chosen by the plain rule) of every densified
    Gaussian with a measured outcome; exploration rows have the flag False."""
    gain, dens = _adjusted_gain(log)
    plain = log.get("plain_dens", torch.ones_like(dens))
    idx = torch.nonzero(dens).flatten()
    return log["feats"][idx], gain[idx], plain[idx]


def offline_gain(mlp: ProposalMLP, outcomes: list, min_gain: float = 0.05) -> dict:
    """Off-policy comparison on logged densifications with measured outcomes,
    one refinement at a time: the plain rule's choices against the network's
    top-K of the same pool (plain + exploration rows) with K = the plain
    count. Reports the mean adjusted held-out gain and the fraction of
    choices reaching `min_gain` for both."""
    tot = {"plain_gain": 0.0, "mlp_gain": 0.0, "plain_hits": 0, "mlp_hits": 0, "chosen": 0}
    for feats, gain, plain in outcomes:
        k = int(plain.sum())
        if k == 0 or feats.shape[0] <= k:
            continue
        z = mlp.logits(mlp.normalise(feats.contiguous()))
        p = torch.softmax(z, dim=1)
        top = torch.topk(p[:, SPLIT] + p[:, CLONE], k).indices
        tot["plain_gain"] += float(gain[plain].sum())
        tot["mlp_gain"] += float(gain[top].sum())
        tot["plain_hits"] += int((gain[plain] >= min_gain).sum())
        tot["mlp_hits"] += int((gain[top] >= min_gain).sum())
        tot["chosen"] += k
    n = max(tot["chosen"], 1)
    return {"chosen": tot["chosen"], "plain_mean_gain": tot["plain_gain"] / n,
            "mlp_mean_gain": tot["mlp_gain"] / n, "plain_hit_rate": tot["plain_hits"] / n,
            "mlp_hit_rate": tot["mlp_hits"] / n}


def labels_from_logs(logs: list, min_gain: float = 0.05, keep_per_step: int = 20_000, seed=0):
    """Training rows for the proposal MLP: raw features, label, weight.

    The outcome of a decision is the relative drop of the per-pixel error that
    the Gaussian (or the rows derived from it) saw over the next window,
    minus the median drop of the kept Gaussians in that window (the drift
    every row sees as training goes on). Densify actions (split / clone) whose
    adjusted drop reaches `min_gain` keep their action as label; those that
    do not become `keep`. Prunes keep `prune`. A random subset of kept rows is
    labelled `keep`. Weights are the adjusted drops' magnitudes (1 for keep /
    prune), so decisions followed by large loss changes count more."""
    g = torch.Generator().manual_seed(seed)
    F, Y, Wt = [], [], []
    for log in logs:
        a = log["action"].to(torch.int64)
        gain, dens = _adjusted_gain(log)
        lab = torch.where(gain >= min_gain, a, torch.full_like(a, KEEP))
        w = gain.abs().clamp(0.05, 2.0)
        idx = torch.nonzero(dens).flatten()
        F.append(log["feats"][idx]); Y.append(lab[idx]); Wt.append(w[idx])
        pr = torch.nonzero(a == PRUNE).flatten()
        if pr.numel():
            pr = pr[torch.randperm(pr.numel(), generator=g)[:keep_per_step].to(pr.device)]
            F.append(log["feats"][pr]); Y.append(a[pr]); Wt.append(torch.ones(pr.numel(), device=pr.device))
        kp = torch.nonzero(a == KEEP).flatten()
        if kp.numel():
            kp = kp[torch.randperm(kp.numel(), generator=g)[:keep_per_step].to(kp.device)]
            F.append(log["feats"][kp]); Y.append(a[kp]); Wt.append(torch.ones(kp.numel(), device=kp.device))
    return (torch.cat(F).contiguous(), torch.cat(Y).to(torch.int32).contiguous(),
            torch.cat(Wt).contiguous())


def merge_samples(samples: list):
    """Concatenates the per-refinement (features, labels, weights) rows."""
    return tuple(torch.cat([s[k] for s in samples]).contiguous() for k in range(3))


def time_to_psnr(history: list, target: float) -> Optional[float]:
    for h in history:
        if h["psnr"] >= target:
            return h["seconds"]
    return None


@dataclass
class ExperimentConfig:
    """The reference's plain rule (ADC-IGS) against the learned proposal on
    the ring-of-views scene."""
    n_gt: int = 500_000
    n_init: int = 100_000
    width: int = 1280
    height: int = 720
    fx: float = 800.0
    iterations: int = 30_000
    densify: DensifyConfig = field(default_factory=DensifyConfig)
    collect_seeds: tuple = (101,)      # scenes whose logged decisions train the network
    offline_seed: Optional[int] = 202  # scene whose logged decisions score it off-policy
    eval_seeds: tuple = (0, 1, 2)      # scenes trained with the plain and learned policies
    explore: float = 1.0
    explore_min: int = 500
    eval_every: int = 250
    fit_rows: int = 2_000_000
    fit_epochs: int = 20
    min_confidence: float = 0.5
    psnr_margin: float = 0.1
    budget_factor: float = 1.0
    igs: "IGS.IgsOptions" = field(default_factory=lambda: IGS.IgsOptions())
    # further learned runs per evaluation scene, one per confidence floor
    # (reported as "learned@<floor>"; 0 = the network picks exactly IGS's counts)
    extra_confidences: tuple = ()


def _balance(labels: torch.Tensor, weights: torch.Tensor) -> torch.Tensor:
    """Scales row weights by the inverse square root of their class's share."""
    w = weights.clone()
    total = float(weights.sum())
    for k in range(4):
        sel = labels == k
        share = float(weights[sel].sum()) / max(total, 1e-12)
        if share > 0:
            w[sel] *= (0.25 / share) ** 0.5
    return w


def collect(cfg: ExperimentConfig, seed: int, device="cuda", log=print):
    """Plain-heuristic run with exploration and decision logging on the
    ring scene of `seed`, up to the end of the densification window."""
    dcfg = cfg.densify
    iters = min(cfg.iterations, cfg.igs.stop + 2 * cfg.igs.every)
    scene = make_ring_scene(cfg.n_gt, width=cfg.width, height=cfg.height, fx=cfg.fx, seed=seed,
                            device=device)
    # the logged run keeps the full run's schedule (decay, growth stop) while
    # stopping right after the densification window
    igs_opts = IGS.IgsOptions(**{**vars(cfg.igs), "iterations": cfg.iterations,
                                 "grow_stop": cfg.igs.growth_stop() if cfg.igs.grow_stop
                                 else max(1, cfg.iterations // 2)})
    tc = TrainConfig(iterations=iters, policy="plain", densify=dcfg, eval_every=iters,
                     seed=seed, explore=cfg.explore, explore_min=cfg.explore_min,
                     log_decisions=True, igs=igs_opts)
    out = train(scene, tc, model=init_from_points(scene, cfg.n_init, seed=seed + 1))
    info = {"seed": seed, "final_psnr": out["history"][-1]["psnr"],
            "gaussians": out["history"][-1]["gaussians"]}
    log(f"collected seed {seed}: {info}")
    return out["samples"], out["outcomes"], info


def fit_proposal(samples: list, cfg: ExperimentConfig, log=print):
    """Fits the proposal MLP on logged rows with its own GPU kernels."""
    F, Y, Wt = merge_samples(samples)
    g = torch.Generator(device=F.device).manual_seed(0)
    if F.shape[0] > cfg.fit_rows:
        idx = torch.randperm(F.shape[0], device=F.device, generator=g)[:cfg.fit_rows]
        F, Y, Wt = F[idx].contiguous(), Y[idx].contiguous(), Wt[idx].contiguous()
    label_counts = [int((Y == k).sum()) for k in range(4)]
    mlp = ProposalMLP(F.device, seed=0)
    mlp.set_normalisation(F)
    Fn = mlp.normalise(F)
    fit_hist = mlp.fit(Fn, Y, _balance(Y, Wt).contiguous(), epochs=cfg.fit_epochs, lr=3e-3,
                       batch=65536)
    acc = float((mlp.logits(Fn).argmax(1).to(torch.int32) == Y).float().mean())
    log(f"mlp fit: rows {F.shape[0]} labels {label_counts} loss {fit_hist[0]:.4f} -> "
        f"{fit_hist[-1]:.4f} acc {acc:.3f}")
    return mlp, {"rows": int(F.shape[0]), "label_counts": label_counts, "fit_loss": fit_hist,
                 "fit_accuracy": acc}


def _summary(h: list, target: float) -> dict:
    return {"time_to_target_s": time_to_psnr(h, target),
            "best_psnr": max(x["psnr"] for x in h), "final_psnr": h[-1]["psnr"],
            "final_gaussians": h[-1]["gaussians"], "train_seconds": h[-1]["seconds"]}


def densify_experiment(cfg: ExperimentConfig, device="cuda", log=print) -> dict:
    """Collect decision logs with the plain rule (ADC-IGS, plus exploration:
    random extra parents) on scenes of other seeds, fit the proposal MLP on
    the GPU with its own kernels, score it off-policy on the logged decisions
    of another scene, then train plain and learned from the same
    initialisation on each evaluation scene and compare the final held-out
    PSNR, the training time to the final model and the model size (and the
    time to the plain run's final PSNR minus `psnr_margin`)."""
    samples, collect_info = [], []
    for s in cfg.collect_seeds:
        smp, _, info = collect(cfg, s, device, log)
        samples += smp
        collect_info.append(info)
        torch.cuda.empty_cache()
    mlp, fit = fit_proposal(samples, cfg, log)
    del samples
    result = {"fit": fit, "collect": collect_info, "mlp": mlp, "seeds": {}}
    if cfg.offline_seed is not None:
        _, outcomes, _ = collect(cfg, cfg.offline_seed, device, log)
        result["offline"] = {**offline_gain(mlp, outcomes), "seed": cfg.offline_seed}
        log(f"offline: {result['offline']}")
        del outcomes
        torch.cuda.empty_cache()
    for seed in cfg.eval_seeds:
        scene = make_ring_scene(cfg.n_gt, width=cfg.width, height=cfg.height, fx=cfg.fx,
                                seed=seed, device=device)
        runs = {}
        variants = [("plain", "plain", cfg.min_confidence), ("learned", "learned",
                                                             cfg.min_confidence)]
        variants += [(f"learned@{c:g}", "learned", c) for c in cfg.extra_confidences]
        for name, policy, conf in variants:
            tc = TrainConfig(iterations=cfg.iterations, policy=policy, densify=cfg.densify,
                             eval_every=cfg.eval_every, seed=seed, igs=cfg.igs,
                             min_confidence=conf, budget_factor=cfg.budget_factor)
            torch.cuda.synchronize()
            out = train(scene, tc, model=init_from_points(scene, cfg.n_init, seed=seed + 1),
                        mlp=mlp if policy == "learned" else None)
            runs[name] = {"history": out["history"], "refinements": out["refinements"]}
            del out
            torch.cuda.empty_cache()
        # Held-out PSNR on this scene family falls from the first evaluation
        # for every policy (the 24 ring views are overfitted), so a threshold
        # below the plain run's quality is met at the start by any run; the
        # comparison is the time to the end of training (the final model) at
        # equal or better final held-out PSNR, with the threshold time kept.
        target = runs["plain"]["history"][-1]["psnr"] - cfg.psnr_margin
        per = {"target_psnr": target}
        for name, r in runs.items():
            per[name] = {**_summary(r["history"], target), "history": r["history"],
                         "refinements": r["refinements"]}
        log(f"seed {seed}: target {target:.3f} " + " ".join(
            f"{n}: ttt {per[n]['time_to_target_s']} best {per[n]['best_psnr']:.3f} "
            f"final {per[n]['final_psnr']:.3f} n {per[n]['final_gaussians']} "
            f"t {per[n]['train_seconds']:.1f}" for n in runs))
        result["seeds"][seed] = per
        del scene
        torch.cuda.empty_cache()
    names = [n for n in result["seeds"][cfg.eval_seeds[0]] if n not in (
        "target_psnr",)]
    ttt = {n: [result["seeds"][s][n]["time_to_target_s"] for s in cfg.eval_seeds]
           for n in names}
    both = [k for k in range(len(cfg.eval_seeds))
            if ttt["plain"][k] is not None and ttt["learned"][k] is not None]
    mean = lambda n, key: (sum(result["seeds"][s][n][key] for s in cfg.eval_seeds)
                           / len(cfg.eval_seeds))
    result["summary"] = {
        "seeds": list(cfg.eval_seeds),
        "learned_reached_target": sum(t is not None for t in ttt["learned"]),
        "learned_faster": sum(ttt["learned"][k] < ttt["plain"][k] for k in both),
        "mean_time_to_target_s": {n: (sum(ttt[n][k] for k in both) / len(both) if both
                                      else None) for n in ttt},
        "mean_best_psnr": {n: mean(n, "best_psnr") for n in ttt},
        "mean_final_psnr": {n: mean(n, "final_psnr") for n in ttt},
        "learned_final_within_margin": sum(
            result["seeds"][s]["learned"]["final_psnr"] >=
            result["seeds"][s]["plain"]["final_psnr"] - cfg.psnr_margin for s in cfg.eval_seeds),
        "mean_train_seconds": {n: mean(n, "train_seconds") for n in ttt},
        "mean_final_gaussians": {n: mean(n, "final_gaussians") for n in ttt},
        "plain_rule": "ADC-IGS (IgsStrategy::refine)",
        "target": f"plain run's final held-out PSNR minus {cfg.psnr_margin} dB",
    }
    return result
