"""Training losses on the library's kernels, through the C ABI: the fused
L1 + SSIM loss photara trains with (photara/src/splat/fused_ssim.cu,
cuda_backend::fused_l1_ssim_loss / fused_ssim_metric) and the whole
per-view training loss around it (cuda_backend::compute_training_loss,
photara/src/splat/cuda_ops.cu:2731)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib as L
from .rasterizer import _pool, _ptr, _require


def _check_image(t: torch.Tensor, name: str) -> None:
    _require(t, name)
    if t.dim() != 3 or t.shape[0] != 3:
        raise ValueError(f"{name} must be [3,H,W]")


def fused_l1_ssim(prediction: torch.Tensor, target: torch.Tensor,
                  mask: Optional[torch.Tensor] = None, ssim_weight: float = 0.2,
                  photometric_weight: float = 1.0, grad: Optional[torch.Tensor] = None):
    """Returns (loss [1] device tensor, grad [3,H,W]): the photometric loss
    w / (3 (W-10)(H-10)) * sum over the valid window of
    [ssim_weight (1 - SSIM) + (1 - ssim_weight) |a - b|] and its gradient with
    respect to `prediction` (added into `grad` when one is given)."""
    _check_image(prediction, "prediction")
    _check_image(target, "target")
    if target.shape != prediction.shape:
        raise ValueError("prediction and target shapes differ")
    H, W = int(prediction.shape[1]), int(prediction.shape[2])
    if mask is not None:
        _require(mask, "mask")
        if mask.numel() != H * W:
            raise ValueError("mask must be [H,W]")
    if grad is None:
        grad = torch.zeros_like(prediction)
    else:
        _check_image(grad, "grad")
    loss = torch.zeros((1,), device=prediction.device)
    ctx = _pool(prediction.device.index or 0).take()
    try:
        ctx.bind_stream()
        L.check(L.load().gs_fused_l1_ssim(ctx.ptr, _ptr(prediction), _ptr(target), _ptr(mask),
                                          W, H, float(ssim_weight), float(photometric_weight),
                                          _ptr(grad), _ptr(loss)), ctx.ptr)
    finally:
        ctx.release()
    return loss, grad


def ssim_metric(prediction: torch.Tensor, target: torch.Tensor,
                mask: Optional[torch.Tensor] = None) -> float:
    """Mean SSIM over the valid window (and the mask's nonzero pixels)."""
    _check_image(prediction, "prediction")
    _check_image(target, "target")
    H, W = int(prediction.shape[1]), int(prediction.shape[2])
    out = torch.zeros((1,), device=prediction.device)
    ctx = _pool(prediction.device.index or 0).take()
    try:
        ctx.bind_stream()
        L.check(L.load().gs_ssim_metric(ctx.ptr, _ptr(prediction), _ptr(target), _ptr(mask),
                                        W, H, _ptr(out)), ctx.ptr)
    finally:
        ctx.release()
    return float(out)


@dataclass
class TrainingLossOptions:
    """Weights of compute_training_loss (photara TrainingOptions /
    TrainingLossSettings defaults). depth_weight and normal_weight are the
    resolved weights of the depth and normal observation terms (0 = off):
    photara resolves them from its MVS / AI-prior switches before the call."""
    photometric_weight: float = 1.0
    ssim_weight: float = 0.2
    depth_weight: float = 0.0
    normal_weight: float = 0.0
    depth_normal_weight: float = 0.0
    match_alpha_weight: float = 0.25
    geometry_epsilon: float = 1e-3
    alpha_mode: str = "masked"  # "masked", "transparent" or "validity"
    ai_prior: bool = False


@dataclass
class LossGradients:
    color: torch.Tensor
    alpha: torch.Tensor
    depth: Optional[torch.Tensor]
    normal: Optional[torch.Tensor]
    terms: Optional[torch.Tensor]  # [4]: rgb, depth, normal, alpha

    @property
    def total(self) -> float:
        return float(self.terms.sum()) if self.terms is not None else float("nan")


_ALPHA_MODES = {"validity": -1, "masked": 0, "transparent": 1}


def compute_training_loss(color: torch.Tensor, target_color: torch.Tensor, *,
                          alpha: Optional[torch.Tensor] = None,
                          median_depth: Optional[torch.Tensor] = None,
                          normal: Optional[torch.Tensor] = None,
                          target_depth: Optional[torch.Tensor] = None,
                          target_normal: Optional[torch.Tensor] = None,
                          mask: Optional[torch.Tensor] = None, camera=None,
                          options: Optional[TrainingLossOptions] = None,
                          collect_scalar_terms: bool = True,
                          need_geometry_gradients: bool = False) -> LossGradients:
    """The training loss of one rendered view and its image gradients
    (cuda_backend::compute_training_loss, photara/src/splat/cuda_ops.cu:2731):
    per-pixel depth, normal and alpha terms, the fused L1 + SSIM colour term
    (plain L1 when the image is 10 pixels or less across), and the
    depth-normal consistency term when `need_geometry_gradients` and
    options.depth_normal_weight > 0 (needs `camera` for the intrinsics).
    The mask, when given, is enabled (photara: has_mask and use_mask)."""
    o = options or TrainingLossOptions()
    _check_image(color, "color")
    _check_image(target_color, "target_color")
    H, W = int(color.shape[1]), int(color.shape[2])
    for t, name, n in ((alpha, "alpha", 1), (median_depth, "median_depth", 1),
                       (normal, "normal", 3), (target_depth, "target_depth", 1),
                       (target_normal, "target_normal", 3), (mask, "mask", 1)):
        if t is not None:
            _require(t, name)
            if t.numel() != n * H * W:
                raise ValueError(f"{name} must hold {n} x {H} x {W} floats")
    if o.alpha_mode not in _ALPHA_MODES:
        raise ValueError(f"alpha_mode must be one of {sorted(_ALPHA_MODES)}")
    dev = color.device
    grads = LossGradients(
        color=torch.empty_like(color), alpha=torch.empty((H, W), device=dev),
        depth=torch.empty((H, W), device=dev) if need_geometry_gradients else None,
        normal=torch.empty((3, H, W), device=dev) if need_geometry_gradients else None,
        terms=torch.zeros((4,), device=dev) if collect_scalar_terms else None)
    im = L.LossImages(_ptr(color), _ptr(alpha), _ptr(median_depth), _ptr(normal),
                      _ptr(target_color), _ptr(target_depth), _ptr(target_normal), _ptr(mask),
                      W, H, *((camera.fx, camera.fy, camera.cx, camera.cy) if camera is not None
                              else (0.0, 0.0, 0.0, 0.0)))
    opt = L.LossOptions(o.photometric_weight, o.ssim_weight, o.depth_weight, o.normal_weight,
                        o.depth_normal_weight, o.match_alpha_weight, o.geometry_epsilon,
                        1 if mask is not None else 0, _ALPHA_MODES[o.alpha_mode],
                        1 if o.ai_prior else 0)
    out = L.LossOutputs(_ptr(grads.color), _ptr(grads.alpha), _ptr(grads.depth),
                        _ptr(grads.normal), _ptr(grads.terms))
    ctx = _pool(dev.index or 0).take()
    try:
        ctx.bind_stream()
        L.check(L.load().gs_training_loss(ctx.ptr, C.byref(im), C.byref(opt), C.byref(out)),
                ctx.ptr)
    finally:
        ctx.release()
    return grads
