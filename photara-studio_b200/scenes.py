"""Seeded synthetic Gaussian scenes with the workload shapes of the benchmark configs.

No public dataset is involved: every scene is drawn from fixed distributions
(means uniform in a box placed in front of the camera, log-scales
N(-3.5, 0.5), quaternions normalised N(0,1)^4, opacity logits N(0,1), SH degree
3 with DC N(0,0.3) and the rest N(0,0.05)).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

IDENTITY16 = [1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0]


@dataclass
class SceneArrays:
    means: np.ndarray           # [N,3] float32
    log_scales: np.ndarray      # [N,3]
    quaternions: np.ndarray     # [N,4]
    opacity_logits: np.ndarray  # [N,1]
    sh: np.ndarray              # [N,16,3]
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    world_to_camera: list
    position: list

    @property
    def count(self) -> int:
        return int(self.means.shape[0])


# name: (N, W, H, f, half_extent_xy, z_lo, z_hi)
CONFIGS = {
    "tiny": (512, 64, 48, 64.0, 1.0, 2.0, 6.0),
    "small": (4096, 128, 96, 128.0, 1.0, 2.0, 6.0),
    "g16k_256": (16384, 256, 256, 256.0, 1.0, 2.0, 6.0),
    "mid": (131072, 640, 480, 500.0, 4.0, 2.0, 12.0),
    "g1m_1080p": (1048576, 1920, 1080, 1500.0, 4.0, 2.0, 12.0),
    "g8m_2160p": (8388608, 3840, 2160, 3000.0, 8.0, 2.0, 30.0),
}


def make_scene(name: str = "g16k_256", seed: int = 0, count: int | None = None) -> SceneArrays:
    n, w, h, f, half, z_lo, z_hi = CONFIGS[name]
    if count is not None:
        n = int(count)
    rng = np.random.default_rng(seed)
    means = np.empty((n, 3), np.float32)
    means[:, 0:2] = rng.uniform(-half, half, size=(n, 2))
    means[:, 2] = rng.uniform(z_lo, z_hi, size=n)
    log_scales = rng.normal(-3.5, 0.5, size=(n, 3)).astype(np.float32)
    q = rng.normal(0.0, 1.0, size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    quats = q.astype(np.float32)
    logits = rng.normal(0.0, 1.0, size=(n, 1)).astype(np.float32)
    sh = np.empty((n, 16, 3), np.float32)
    sh[:, 0, :] = rng.normal(0.0, 0.3, size=(n, 3))
    sh[:, 1:, :] = rng.normal(0.0, 0.05, size=(n, 15, 3))
    return SceneArrays(means, log_scales, quats, logits, sh, w, h, f, f, w / 2.0, h / 2.0,
                       list(IDENTITY16), [0.0, 0.0, 0.0])


def perturbed_target_means(scene: SceneArrays, seed: int = 1, sigma: float = 0.01) -> np.ndarray:
    """Means of the L1 target render: the scene's means + N(0, sigma)."""
    rng = np.random.default_rng(seed)
    return (scene.means + rng.normal(0.0, sigma, size=scene.means.shape)).astype(np.float32)


# Resolutions of the batched multi-view workload.
BATCH_SIZES = ((640, 480), (1280, 720), (1600, 1200), (1920, 1080))


@dataclass
class RingView:
    eye: tuple
    width: int
    height: int
    focal: float


def make_ring_batch(count: int, views: int = 32, sizes=BATCH_SIZES, radius: float = 6.0,
                    half: float = 2.0, seed: int = 0, fov_deg: float = 90.0):
    """Gaussians with the distributions above, means uniform in [-half, half]^3
    around the origin, and `views` cameras on a ring of `radius` (height 0.5)
    looking at the origin, each with a resolution drawn uniformly from `sizes`
    and a horizontal field of view of `fov_deg`."""
    rng = np.random.default_rng(seed)
    n = int(count)
    means = rng.uniform(-half, half, size=(n, 3)).astype(np.float32)
    log_scales = rng.normal(-3.5, 0.5, size=(n, 3)).astype(np.float32)
    q = rng.normal(0.0, 1.0, size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    logits = rng.normal(0.0, 1.0, size=(n, 1)).astype(np.float32)
    sh = np.empty((n, 16, 3), np.float32)
    sh[:, 0, :] = rng.normal(0.0, 0.3, size=(n, 3))
    sh[:, 1:, :] = rng.normal(0.0, 0.05, size=(n, 15, 3))
    arrays = SceneArrays(means, log_scales, q.astype(np.float32), logits, sh, 0, 0, 0.0, 0.0,
                         0.0, 0.0, list(IDENTITY16), [0.0, 0.0, 0.0])
    picks = rng.integers(0, len(sizes), size=views)
    tan_half = np.tan(np.radians(fov_deg) / 2.0)
    ring = []
    for k in range(views):
        a = 2.0 * np.pi * k / views
        w, h = sizes[int(picks[k])]
        ring.append(RingView((radius * np.cos(a), 0.5, radius * np.sin(a)), int(w), int(h),
                             float(w / (2.0 * tan_half))))
    return arrays, ring
