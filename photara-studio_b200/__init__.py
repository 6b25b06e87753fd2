"""B200-native (sm_100a) 3D Gaussian Splatting rasterizer.

Drop-in for the forward/backward path that photara's splat trainer calls into
its splat_drender backend. The compute lives in libgsplat_b200.so (C ABI,
include/gsplat_b200.h); this package is the host-side mirror of photara's
Rasterizer interface plus the autograd wrapper.
"""
from . import _lib
from .rasterizer import (Camera, GaussianModel, ModelGradients, RasterizationPolicy,
                         RasterizeOptions, Rasterizer, RenderResult, SHAdamUpdate,
                         StructureAdamUpdate, draw_list, look_at_camera, stage_times)
from .autograd import RasterizeGaussians, rasterize_gaussians
from .scenes import make_scene
from .loss import (LossGradients, TrainingLossOptions, compute_training_loss, fused_l1_ssim,
                   ssim_metric)
from . import densify, trainer

__all__ = [
    "Camera", "GaussianModel", "ModelGradients", "RasterizationPolicy", "RasterizeOptions",
    "Rasterizer", "RenderResult", "SHAdamUpdate", "StructureAdamUpdate", "draw_list",
    "look_at_camera", "stage_times", "make_scene", "load_library", "RasterizeGaussians",
    "rasterize_gaussians", "densify", "trainer", "fused_l1_ssim", "ssim_metric",
    "compute_training_loss", "TrainingLossOptions", "LossGradients",
]


def load_library():
    """Loads libgsplat_b200.so (raises when it has not been built)."""
    return _lib.load()
