"""torch.autograd.Function over the hand-written forward / adjoint.

`rasterize_gaussians` renders one view and, in backward, runs the library's
reverse-order adjoint (per-tile recomputation of transmittance from the stored
final T, no per-pixel lists) and returns gradients with respect to the raw
parameters (means, log-scales, quaternions, opacity logits, SH), so the usual
torch optimisers and `torch.autograd.gradcheck` apply. The fused-Adam training
path stays on `Rasterizer.backward(..., structure_adam=, sh_adam=)`.
"""
from __future__ import annotations

from typing import Optional

import torch

from .rasterizer import Camera, GaussianModel, RasterizeOptions, Rasterizer


class RasterizeGaussians(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, log_scales, quaternions, opacity_logits, sh, camera: Camera,
                options: RasterizeOptions, sh_degree: int):
        model = GaussianModel(means.detach().contiguous(), log_scales.detach().contiguous(),
                              quaternions.detach().contiguous(),
                              opacity_logits.detach().contiguous(), sh.detach().contiguous(),
                              sh_degree)
        rendered = Rasterizer().forward(model, camera, options)
        ctx.model = model
        ctx.rendered = rendered
        ctx.logit_shape = opacity_logits.shape
        ctx.mark_non_differentiable(rendered.radii)
        return rendered.color, rendered.alpha, rendered.radii

    @staticmethod
    def backward(ctx, grad_color, grad_alpha, _grad_radii):
        if grad_color is None:
            grad_color = torch.zeros_like(ctx.rendered.color)
        g = Rasterizer().backward(ctx.model, ctx.rendered, grad_color.contiguous(),
                                  None if grad_alpha is None else grad_alpha.contiguous())
        return (g.means, g.log_scales, g.quaternions, g.opacity_logits.view(ctx.logit_shape),
                g.sh, None, None, None)


def rasterize_gaussians(means: torch.Tensor, log_scales: torch.Tensor, quaternions: torch.Tensor,
                        opacity_logits: torch.Tensor, sh: torch.Tensor, camera: Camera,
                        options: Optional[RasterizeOptions] = None, sh_degree: int = 3):
    """Differentiable render of one pinhole view: returns (color [3,H,W], alpha [H,W], radii [N])."""
    options = options or RasterizeOptions(active_sh_degree=sh_degree)
    return RasterizeGaussians.apply(means, log_scales, quaternions, opacity_logits, sh, camera,
                                    options, sh_degree)
