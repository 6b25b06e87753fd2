"""Photometric losses on the library's kernels: the fused L1 + SSIM loss
photara trains with (photara/src/splat/fused_ssim.cu,
cuda_backend::fused_l1_ssim_loss / fused_ssim_metric), through the C ABI."""
from __future__ import annotations

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
