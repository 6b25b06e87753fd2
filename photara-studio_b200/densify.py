"""Adaptive density control: plain heuristic and learned proposal MLP.

Statistics, decisions, features, the split and the MLP run as hand-written
kernels through the C ABI (csrc/densify.cu, csrc/mlp.cu); this module keeps the
tensors and applies a decision (prune / split / clone) to the model and its
Adam state. Follows the reference's densification data flow
(photara/src/splat/trainer.cpp:2441 statistics after each backward,
photara/src/splat/densification.cpp refine schedule, cuda_ops.cu:1548-1845).

Actions: 0 keep, 1 split, 2 clone, 3 prune.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional

import torch

from . import _lib as L
from .rasterizer import GaussianModel, _pool

KEEP, SPLIT, CLONE, PRUNE = 0, 1, 2, 3
N_FEATURES = 8


def _p(t):
    return None if t is None else t.data_ptr()


class _Ctx:
    """A native context borrowed for densification launches on the current stream."""

    def __init__(self, device: int):
        self.ctx = _pool(device).take()

    def __enter__(self):
        self.ctx.bind_stream()
        return self.ctx.ptr

    def __exit__(self, *exc):
        self.ctx.release()


@dataclass
class DensifyConfig:
    grad_threshold: float = 2.0e-4
    percent_dense: float = 0.01
    prune_opacity: float = 1.0 / 255.0
    prune_world_scale: float = 0.1
    prune_screen: float = 0.25       # max screen radius / max(W, H) (quarter frame)
    start: int = 500
    every: int = 100
    stop: int = 15_000
    opacity_reset_every: int = 3_000
    cap: int = 3_000_000


class DensifyStats:
    """Per-Gaussian statistics between refinements (gs_densify_stats)."""

    NAMES = ("grad_acc", "count", "max_screen", "err_num", "err_den", "depth_acc", "age")

    def __init__(self, n: int, device):
        self.t = {k: torch.zeros(n, device=device) for k in self.NAMES}

    def struct(self) -> L.DensifyStats:
        return L.DensifyStats(*[_p(self.t[k]) for k in self.NAMES])

    def accumulate(self, rendered, grads, camera, means: torch.Tensor) -> None:
        """Adds one view; `camera` supplies the view-space depth row and the
        resolution that normalises screen radii."""
        n = rendered.radii.numel()
        w = [float(v) for v in camera.world_to_camera]  # column-major 4x4
        row = (C.c_float * 4)(w[2], w[6], w[10], w[14])
        with _Ctx(rendered.radii.device.index or 0) as ctx:
            L.check(L.load().gs_densify_accumulate(
                ctx, n, _p(grads.refine_weight), _p(rendered.radii), _p(grads.densify_weight),
                _p(grads.densify_weight_den), 1.0 / max(camera.width, camera.height),
                _p(means), row, C.byref(self.struct())), ctx)

    def reset(self, keep_age: bool = True) -> None:
        for k in self.NAMES:
            if k != "age" or not keep_age:
                self.t[k].zero_()

    def remap(self, index: torch.Tensor, n_new_children: int) -> None:
        """Rows follow the model: `index` selects survivors, children start fresh."""
        for k in self.NAMES:
            kept = self.t[k].index_select(0, index)
            self.t[k] = torch.cat([kept, torch.zeros(n_new_children, device=kept.device)])


def adc_decide(model: GaussianModel, stats: DensifyStats, cfg: DensifyConfig, extent: float,
               densify: bool = True, prune_screen: bool = True) -> torch.Tensor:
    """Plain ADC action per Gaussian; `prune_screen` enables the screen-size
    prune (the classic rule applies it only after the first opacity reset)."""
    n = model.size()
    action = torch.empty(n, dtype=torch.int32, device=model.means.device)
    p = L.AdcParams(cfg.grad_threshold, cfg.percent_dense, extent, cfg.prune_opacity,
                    cfg.prune_world_scale, cfg.prune_screen if prune_screen else 0.0,
                    1 if densify else 0)
    with _Ctx(model.means.device.index or 0) as ctx:
        L.check(L.load().gs_adc_decide(ctx, n, _p(model.log_scales), _p(model.opacity_logits),
                                       C.byref(stats.struct()), C.byref(p), _p(action)), ctx)
    return action


def features(model: GaussianModel, stats: DensifyStats, center, extent: float,
             norm: Optional[torch.Tensor] = None) -> torch.Tensor:
    n = model.size()
    out = torch.empty((n, N_FEATURES), device=model.means.device)
    c3 = (C.c_float * 3)(*[float(v) for v in center])
    with _Ctx(model.means.device.index or 0) as ctx:
        L.check(L.load().gs_densify_features(
            ctx, n, _p(model.means), _p(model.log_scales), _p(model.opacity_logits), _p(model.sh),
            int(model.sh.shape[1]) * 3, C.byref(stats.struct()), c3, float(extent), _p(norm),
            _p(out)), ctx)
    return out


class ProposalMLP:
    """8 -> 64 -> 64 -> 4 MLP with BF16 weights (FP32 master copy), FP32 accumulation."""

    def __init__(self, device, seed: int = 0):
        self.device = torch.device(device)
        n = L.load().gs_mlp_param_count()
        g = torch.Generator().manual_seed(seed)
        w = torch.zeros(n)
        # He-style init per layer (layout W1[8][64] b1[64] W2[64][64] b2[64] W3[64][4] b3[4])
        w[:512] = torch.randn(512, generator=g) * math.sqrt(2.0 / 8)
        w[576:576 + 4096] = torch.randn(4096, generator=g) * math.sqrt(2.0 / 64)
        w[4736:4736 + 256] = torch.randn(256, generator=g) * math.sqrt(1.0 / 64)
        self.master = w.to(self.device)
        self.bf16 = self.master.to(torch.bfloat16)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.step = 0
        self.norm = torch.cat([torch.zeros(N_FEATURES), torch.ones(N_FEATURES)]).to(self.device)

    def set_normalisation(self, raw_features: torch.Tensor) -> None:
        mean = raw_features.mean(0)
        std = raw_features.std(0).clamp_min(1e-6)
        self.norm = torch.cat([mean, 1.0 / std]).contiguous()

    def normalise(self, raw: torch.Tensor) -> torch.Tensor:
        return ((raw - self.norm[:N_FEATURES]) * self.norm[N_FEATURES:]).contiguous()

    def logits(self, feats: torch.Tensor) -> torch.Tensor:
        n = feats.shape[0]
        out = torch.empty((n, 4), device=self.device)
        with _Ctx(self.device.index or 0) as ctx:
            L.check(L.load().gs_mlp_forward(ctx, n, _p(feats), _p(self.bf16), _p(out)), ctx)
        return out

    def loss_and_grad(self, feats, labels, weights):
        grad = torch.zeros_like(self.master)
        loss = torch.zeros(1, device=self.device)
        with _Ctx(self.device.index or 0) as ctx:
            L.check(L.load().gs_mlp_train_step(
                ctx, feats.shape[0], _p(feats), _p(labels), _p(weights), _p(self.bf16),
                float(weights.sum()), _p(grad), _p(loss)), ctx)
        return float(loss.item()), grad

    def adam_step(self, grad, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8) -> None:
        self.step += 1
        with _Ctx(self.device.index or 0) as ctx:
            L.check(L.load().gs_mlp_adam(ctx, _p(self.master), _p(self.bf16), _p(grad),
                                         _p(self.m), _p(self.v), lr, b1, b2,
                                         1 - b1 ** self.step, 1 - b2 ** self.step, eps), ctx)

    def fit(self, feats, labels, weights, epochs=200, lr=3e-3, batch=65536, seed=0) -> list:
        """Full-batch-ish training on logged samples (minibatches of `batch` rows)."""
        n = feats.shape[0]
        g = torch.Generator(device=self.device).manual_seed(seed)
        history = []
        for _ in range(epochs):
            perm = torch.randperm(n, device=self.device, generator=g)
            tot = 0.0
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                loss, grad = self.loss_and_grad(feats[idx].contiguous(),
                                                labels[idx].contiguous(),
                                                weights[idx].contiguous())
                self.adam_step(grad, lr=lr)
                tot += loss
            history.append(tot)
        return history

    def propose(self, feats_raw: torch.Tensor, fallback: torch.Tensor, stats: DensifyStats,
                min_confidence: float = 0.5) -> torch.Tensor:
        z = self.logits(self.normalise(feats_raw))
        out = torch.empty_like(fallback)
        with _Ctx(self.device.index or 0) as ctx:
            L.check(L.load().gs_proposal_policy(ctx, fallback.numel(), _p(z), _p(fallback),
                                                C.byref(stats.struct()), float(min_confidence),
                                                _p(out)), ctx)
        return out

    def propose_budget(self, feats_raw: torch.Tensor, fallback: torch.Tensor,
                       stats: DensifyStats, budget: int,
                       min_confidence: float = 0.5) -> torch.Tensor:
        """Learned proposal with a growth cap.

        Per Gaussian the proposal kernel takes the network's argmax where its
        softmax confidence reaches min_confidence and the plain heuristic's
        decision elsewhere (fallback); the plain rule's hard prunes always
        apply and densification needs a Gaussian the statistics saw. When the
        network proposes more than `budget` densifications, only the `budget`
        with the highest p(split) + p(clone) are kept (the rest keep)."""
        z = self.logits(self.normalise(feats_raw))
        out = torch.empty_like(fallback)
        with _Ctx(self.device.index or 0) as ctx:
            L.check(L.load().gs_proposal_policy(ctx, fallback.numel(), _p(z), _p(fallback),
                                                C.byref(stats.struct()), float(min_confidence),
                                                _p(out)), ctx)
        p = torch.softmax(z, dim=1)
        confident = p.max(dim=1).values >= min_confidence
        mlp_dens = confident & ((out == SPLIT) | (out == CLONE))
        extra = int(mlp_dens.sum()) - max(int(budget), 0)
        if extra > 0:
            score = torch.where(mlp_dens, p[:, SPLIT] + p[:, CLONE],
                                torch.full_like(p[:, 0], 3.0))
            drop = torch.topk(score, extra, largest=False).indices
            out[drop] = KEEP
        return out

    def state_dict(self):
        return {"master": self.master.cpu(), "norm": self.norm.cpu()}

    def load_state_dict(self, d):
        self.master = d["master"].to(self.device)
        self.bf16 = self.master.to(torch.bfloat16)
        self.norm = d["norm"].to(self.device)


@dataclass
class AdamState:
    """Fused-Adam state of a model (structure FP32 moments + quantized SH)."""
    structure: dict = field(default_factory=dict)
    sh: dict = field(default_factory=dict)

    @staticmethod
    def zeros(model: GaussianModel) -> "AdamState":
        z = torch.zeros_like
        st = AdamState()
        st.structure = dict(means_first=z(model.means), means_second=z(model.means),
                            scales_first=z(model.log_scales), scales_second=z(model.log_scales),
                            rotations_first=z(model.quaternions),
                            rotations_second=z(model.quaternions),
                            opacity_first=z(model.opacity_logits),
                            opacity_second=z(model.opacity_logits))
        st.sh = dict(first=torch.zeros(model.sh.shape, dtype=torch.float16,
                                       device=model.sh.device),
                     packed=torch.zeros(model.sh.shape, dtype=torch.uint8, device=model.sh.device),
                     bounds=torch.zeros((model.size(), 4), device=model.sh.device))
        return st


SPLIT_MODES = {"adc_covariance": 0, "dense_tangent": 1, "igs_random": 2, "long_axis": 3}


def select_rows(keep: torch.Tensor) -> torch.Tensor:
    """Indices (int32, increasing) of the rows whose keep flag is set: the
    library's stable compaction (gs_select_rows); one count read-back."""
    if keep.dtype == torch.bool:
        keep = keep.view(torch.uint8)
    if keep.dtype != torch.uint8 or not keep.is_cuda or not keep.is_contiguous():
        raise ValueError("keep must be a contiguous CUDA bool/uint8 vector")
    n = keep.numel()
    idx = torch.empty((max(n, 1),), dtype=torch.int32, device=keep.device)
    count = torch.zeros((1,), dtype=torch.int32, device=keep.device)
    with _Ctx(keep.device.index or 0) as ctx:
        L.check(L.load().gs_select_rows(ctx, n, _p(keep), _p(idx), _p(count)), ctx)
    return idx[:int(count.item())]


def gather_rows(indices: torch.Tensor, arrays: list, rows: Optional[int] = None) -> list:
    """New tensors whose row i is row indices[i] of each array (one launch for
    all arrays, gs_gather_rows). With `rows` > len(indices) the extra tail
    rows are zero (new Adam moments)."""
    if indices.dtype != torch.int32 or not indices.is_contiguous():
        raise ValueError("indices must be contiguous int32")
    count = indices.numel()
    rows = count if rows is None else rows
    outs = []
    for a in arrays:
        if not a.is_contiguous() or not a.is_cuda:
            raise ValueError("gather arrays must be contiguous CUDA tensors")
        shape = (rows,) + tuple(a.shape[1:])
        outs.append(torch.zeros(shape, dtype=a.dtype, device=a.device) if rows > count
                    else torch.empty(shape, dtype=a.dtype, device=a.device))
    if count == 0 or not arrays:
        return outs
    for start in range(0, len(arrays), 32):
        part = list(range(start, min(start + 32, len(arrays))))
        k = len(part)
        src = (C.c_void_p * k)(*[arrays[i].data_ptr() for i in part])
        dst = (C.c_void_p * k)(*[outs[i].data_ptr() for i in part])
        row_bytes = (C.c_size_t * k)(*[arrays[i][0].numel() * arrays[i].element_size()
                                       if arrays[i].shape[0] else 4 for i in part])
        with _Ctx(indices.device.index or 0) as ctx:
            L.check(L.load().gs_gather_rows(ctx, count, _p(indices), k, src, dst, row_bytes),
                    ctx)
    return outs


def split_gaussians(parents: GaussianModel, children: GaussianModel, parent_indices: torch.Tensor,
                    mode: str = "adc_covariance", random_samples: Optional[torch.Tensor] = None,
                    screen_sizes: Optional[torch.Tensor] = None, minimum_opacity: float = 1e-6,
                    split_at_screen_size: float = 0.0, split_opacity_k: float = 0.5) -> None:
    """photara's cuda_backend::split_gaussians (cuda_ops.cu:3105): parent rows
    parent_indices[k] move by -offset, child row k (whose log scales hold its
    parent's) lands at +offset; both take the mode's opacity. In place."""
    count = parent_indices.numel()
    if count == 0:
        return
    if mode not in SPLIT_MODES:
        raise ValueError(f"mode must be one of {sorted(SPLIT_MODES)}")
    a = L.SplitArgs(_p(parents.means), _p(parents.log_scales), _p(parents.opacity_logits),
                    _p(parents.quaternions), _p(children.means), _p(children.log_scales),
                    _p(children.opacity_logits), _p(parent_indices), _p(random_samples),
                    _p(screen_sizes), count, SPLIT_MODES[mode], float(minimum_opacity),
                    float(split_at_screen_size), float(split_opacity_k))
    with _Ctx(parents.means.device.index or 0) as ctx:
        L.check(L.load().gs_split_gaussians_mode(ctx, C.byref(a)), ctx)


def apply_adc_decay(model: GaussianModel, opacity_decay: float, scale_decay: float) -> None:
    """photara's cuda_backend::apply_adc_decay (cuda_ops.cu:3388), in place."""
    with _Ctx(model.means.device.index or 0) as ctx:
        L.check(L.load().gs_adc_decay(ctx, model.size(), _p(model.log_scales),
                                      _p(model.opacity_logits), float(opacity_decay),
                                      float(scale_decay)), ctx)


def select_training_rows(model: GaussianModel, adam: "AdamState",
                         keep: torch.Tensor) -> tuple[GaussianModel, "AdamState"]:
    """Prune to the kept rows, parameters and every Adam moment (structure
    FP32, quantized SH) together (select_training_rows_gpu,
    densification_adc_plus.cpp:68-77): one compaction, one gather launch."""
    idx = select_rows(keep)
    fields = ("means", "log_scales", "quaternions", "opacity_logits", "sh")
    s_keys, h_keys = list(adam.structure), list(adam.sh)
    arrays = ([getattr(model, f) for f in fields] + [adam.structure[k] for k in s_keys] +
              [adam.sh[k] for k in h_keys])
    out = gather_rows(idx, arrays)
    m2 = GaussianModel(*out[:5], model.sh_degree)
    a2 = AdamState()
    a2.structure = dict(zip(s_keys, out[5:5 + len(s_keys)]))
    a2.sh = dict(zip(h_keys, out[5 + len(s_keys):]))
    return m2, a2


def apply_actions(model: GaussianModel, adam: AdamState, stats: DensifyStats,
                  action: torch.Tensor, cap: int) -> tuple[GaussianModel, AdamState, dict]:
    """Prune / split / clone rows. Survivors keep their Adam state; new rows
    (children and clones) start with zero moments; the cap limits growth
    (the highest-gradient candidates win)."""
    dev = model.means.device
    n = model.size()
    prune = action == PRUNE
    split = torch.nonzero(action == SPLIT).flatten()
    clone = torch.nonzero(action == CLONE).flatten()
    keep_mask = ~prune
    survivors = int(keep_mask.sum())
    room = max(cap - survivors, 0)
    if split.numel() + clone.numel() > room:
        cand = torch.cat([split, clone])
        kind = torch.cat([torch.ones_like(split), torch.zeros_like(clone)])
        score = stats.t["grad_acc"][cand] / stats.t["count"][cand].clamp_min(1)
        order = torch.argsort(score, descending=True)[:room]
        cand, kind = cand[order], kind[order]
        split, clone = cand[kind == 1], cand[kind == 0]
    split = split[keep_mask[split]]
    clone = clone[keep_mask[clone]]
    # survivors first (order preserved), then split children, then clones
    survivors_idx = select_rows(keep_mask.contiguous())
    new_rows = torch.cat([split, clone]).to(torch.int32)
    gather = torch.cat([survivors_idx, new_rows]).contiguous()
    fields = ("means", "log_scales", "quaternions", "opacity_logits", "sh")
    m2 = GaussianModel(*gather_rows(gather, [getattr(model, f) for f in fields]),
                       model.sh_degree)
    # parents of split children at their new (compacted) positions
    if split.numel():
        remap = torch.full((n,), -1, dtype=torch.int32, device=dev)
        remap[survivors_idx.long()] = torch.arange(survivors_idx.numel(), dtype=torch.int32,
                                                   device=dev)
        parents = remap[split].contiguous()
        with _Ctx(dev.index or 0) as ctx:
            L.check(L.load().gs_split_gaussians(ctx, int(split.numel()), _p(parents),
                                                int(survivors_idx.numel()), _p(m2.means),
                                                _p(m2.log_scales), _p(m2.quaternions),
                                                _p(m2.opacity_logits)), ctx)
    n_new = int(new_rows.numel())
    # survivors keep their moments, new rows start from zero: one gather
    s_keys, h_keys = list(adam.structure), list(adam.sh)
    moved = gather_rows(survivors_idx, [adam.structure[k] for k in s_keys] +
                        [adam.sh[k] for k in h_keys], rows=survivors_idx.numel() + n_new)
    a2 = AdamState()
    a2.structure = dict(zip(s_keys, moved[:len(s_keys)]))
    a2.sh = dict(zip(h_keys, moved[len(s_keys):]))
    stats.remap(survivors_idx.to(torch.int64), n_new)
    info = {"pruned": int(prune.sum()), "split": int(split.numel()),
            "cloned": int(clone.numel()), "count": m2.size(), "gather": gather}
    return m2, a2, info


def reset_opacity(model: GaussianModel, ceiling: float = 0.01) -> None:
    """Classic opacity reset: clamp every opacity to at most `ceiling`."""
    logit = math.log(ceiling / (1 - ceiling))
    model.opacity_logits.clamp_(max=logit)
