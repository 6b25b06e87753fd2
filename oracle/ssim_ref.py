"""Float64 NumPy restatement of the fused L1 + SSIM photometric loss and its
gradient (photara/src/splat/fused_ssim.cu, the loss photara trains with).

TEST INFRASTRUCTURE ONLY: the checker for the library's fused loss kernel,
used by tests/; never by the product.

SSIM of Wang, Bovik, Sheikh and Simoncelli (2004): per channel, local means,
variances and covariance under an 11 x 11 separable Gaussian window (sigma
1.5, zero padding outside the image), C1 = 0.01^2, C2 = 0.03^2. With
lambda = ssim_weight, the loss is
    L = w / (3 (W - 10) (H - 10)) * sum over channels and over the pixels whose
        window lies inside the image of [lambda (1 - SSIM) + (1 - lambda) |a - b|]
(w = photometric_weight; a, b = prediction and target, each times the mask
when one is given), and the gradient is dL/d prediction (times the mask).
"""
from __future__ import annotations

import numpy as np

# The 11-tap window as float32 values (fused_ssim.cu:25-28).
WINDOW = np.array([0.001028380123898387, 0.0075987582094967365, 0.036000773310661316,
                   0.10936068743467331, 0.21300552785396576, 0.26601171493530273,
                   0.21300552785396576, 0.10936068743467331, 0.036000773310661316,
                   0.0075987582094967365, 0.001028380123898387], np.float64)
C1 = 0.01 ** 2
C2 = 0.03 ** 2
HALO = 5


def _blur(x: np.ndarray) -> np.ndarray:
    """Separable window filter with zero padding, same size (last two axes)."""
    H, W = x.shape[-2:]
    p = np.pad(x, [(0, 0)] * (x.ndim - 2) + [(HALO, HALO), (HALO, HALO)])
    h = sum(WINDOW[d] * p[..., :, d:d + W] for d in range(2 * HALO + 1))
    return sum(WINDOW[d] * h[..., d:d + H, :] for d in range(2 * HALO + 1))


def fused_l1_ssim(pred, target, mask=None, ssim_weight=0.2, photometric_weight=1.0):
    """Returns (loss, grad [3,H,W], ssim map [3,H,W]) in float64."""
    a = np.asarray(pred, np.float64)
    b = np.asarray(target, np.float64)
    m = None if mask is None else np.asarray(mask, np.float64)
    if m is not None:
        a, b = a * m, b * m
    C, H, W = a.shape
    lam = float(ssim_weight)
    mu1, mu2 = _blur(a), _blur(b)
    s11, s22, s12 = _blur(a * a) - mu1 * mu1, _blur(b * b) - mu2 * mu2, _blur(a * b) - mu1 * mu2
    A = mu1 * mu1 + mu2 * mu2 + C1
    B = s11 + s22 + C2
    Cn = 2 * mu1 * mu2 + C1
    D = 2 * s12 + C2
    ssim = Cn * D / (A * B)
    valid = np.zeros((H, W), bool)
    valid[HALO:H - HALO, HALO:W - HALO] = True
    norm = float(photometric_weight) / (C * (W - 2 * HALO) * (H - 2 * HALO))
    chain = np.where(valid, norm, 0.0)
    loss = float(((lam * (1 - ssim) + (1 - lam) * np.abs(a - b)) * chain).sum())
    # d SSIM / d (mu1, sigma1^2, sigma12), the mean-subtraction terms folded
    # into d/d mu1 as in the reference's three maps
    dm_dmu1 = (2 * mu2 * D) / (A * B) - (2 * mu2 * Cn) / (A * B) \
        - (2 * mu1 * Cn * D) / (A * A * B) + (2 * mu1 * Cn * D) / (A * B * B)
    dm_ds11 = -Cn * D / (A * B * B)
    dm_ds12 = 2 * Cn / (A * B)
    g0 = _blur(-lam * dm_dmu1 * chain)
    g1 = _blur(-lam * dm_ds11 * chain)
    g2 = _blur(-lam * dm_ds12 * chain)
    sign = np.sign(a - b)
    grad = g0 + 2 * a * g1 + b * g2 + (1 - lam) * sign * chain
    if m is not None:
        grad = grad * m
    return loss, grad, ssim


def ssim_metric(pred, target, mask=None) -> float:
    """Mean SSIM over the valid window (and the mask's nonzero pixels)."""
    _, _, ssim = fused_l1_ssim(pred, target, mask, 1.0, 1.0)
    C, H, W = ssim.shape
    keep = np.zeros((H, W), bool)
    keep[HALO:H - HALO, HALO:W - HALO] = True
    if mask is not None:
        keep &= np.asarray(mask) > 0
    n = int(keep.sum()) * C
    return float(ssim[:, keep].sum() / n) if n else 0.0
