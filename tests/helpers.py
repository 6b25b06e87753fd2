"""Shared test helpers: device models from seeded scenes."""
from __future__ import annotations

import importlib

import numpy as np
import torch

gsb = importlib.import_module("photara-studio_b200")


def device_model(scene, device="cuda", means=None):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
    return gsb.GaussianModel(
        means=t(scene.means if means is None else means), log_scales=t(scene.log_scales),
        quaternions=t(scene.quaternions), opacity_logits=t(scene.opacity_logits), sh=t(scene.sh),
        sh_degree=3)


def camera_of(scene):
    return gsb.Camera(scene.world_to_camera, scene.position, scene.fx, scene.fy, scene.cx,
                      scene.cy, scene.width, scene.height)


def clone_model(m):
    return gsb.GaussianModel(m.means.clone(), m.log_scales.clone(), m.quaternions.clone(),
                             m.opacity_logits.clone(), m.sh.clone(), m.sh_degree,
                             None if m.filter_3d is None else m.filter_3d.clone())
