"""Fused L1 + SSIM loss and the SSIM metric (photara/src/splat/fused_ssim.cu)
on the library's kernel, against the reference's own test values
(photara/tests/splat_test.cpp: test_ssim_loss, test_ssim_loss_large_reduction,
test_ssim_metric_large_reduction) and the float64 restatement
(oracle/ssim_ref.py)."""
import numpy as np
import pytest
import torch

from helpers import gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]

S = pytest.importorskip("oracle.ssim_ref")


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def test_matches_reference_test_values():
    """13 x 13, one bright pixel, ssim_weight 1 (splat_test.cpp test_ssim_loss):
    loss 0.299324721, centre gradient 0.152631640, gradient sum 0.004020121,
    absolute sum 0.301243156, each within 2e-5."""
    side = 13
    pred = np.full((3, side, side), 0.4, np.float32)
    tgt = np.full((3, side, side), 0.4, np.float32)
    pred[0, 6, 6] = 0.8
    loss, grad = gsb.fused_l1_ssim(_t(pred), _t(tgt), None, ssim_weight=1.0)
    g = grad.cpu().numpy().ravel()
    assert abs(float(loss) - 0.299324721) < 2e-5
    assert abs(g[6 * side + 6] - 0.152631640) < 2e-5
    assert abs(float(g.sum()) - 0.004020121) < 2e-5, float(g.sum())
    assert abs(float(np.abs(g).sum()) - 0.301243156) < 2e-5, float(np.abs(g).sum())


def test_constant_images_large_reduction():
    """2051 x 1027 constant images (test_ssim_loss_large_reduction): the loss
    is 0.8 (r - p) + 0.2 (1 - SSIM) within 3e-5; reporting the loss does not
    change the gradient."""
    W, H, p, r = 2051, 1027, 0.25, 0.75
    pred = torch.full((3, H, W), p, device="cuda")
    tgt = torch.full((3, H, W), r, device="cuda")
    loss, g1 = gsb.fused_l1_ssim(pred, tgt, None, 0.2, 1.0)
    ssim = (2 * p * r + 1e-4) / (p * p + r * r + 1e-4)
    assert abs(float(loss) - (0.8 * (r - p) + 0.2 * (1 - ssim))) < 3e-5
    lib = gsb.load_library()
    ctx = gsb.rasterizer._pool(0).take()
    ctx.bind_stream()
    g2 = torch.zeros_like(pred)
    assert lib.gs_fused_l1_ssim(ctx.ptr, pred.data_ptr(), tgt.data_ptr(), None, W, H, 0.2, 1.0,
                                g2.data_ptr(), None) == 0
    torch.cuda.synchronize()
    ctx.release()
    assert torch.equal(g1, g2)


@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("size", [(97, 61), (1920, 1080)])
def test_matches_float64_oracle(masked, size):
    W, H = size
    rng = np.random.default_rng(W + masked)
    tgt = rng.uniform(0.1, 0.9, (3, H, W)).astype(np.float32)
    pred = np.clip(tgt + rng.normal(0, 0.08, tgt.shape), 0, 1).astype(np.float32)
    mask = (rng.uniform(size=(H, W)) > 0.3).astype(np.float32) if masked else None
    loss, grad = gsb.fused_l1_ssim(_t(pred), _t(tgt), None if mask is None else _t(mask),
                                   0.2, 0.7)
    lo, go, _ = S.fused_l1_ssim(pred, tgt, mask, 0.2, 0.7)
    assert abs(float(loss) - lo) <= 1e-5 * abs(lo)
    g = grad.cpu().numpy().astype(np.float64)
    scale = np.abs(go).max()
    assert np.abs(g - go).max() <= 1e-4 * scale, np.abs(g - go).max() / scale
    # the loss adds into the caller's scalar (cuda_backend::fused_l1_ssim_loss
    # scalar_terms), the gradient into a given buffer
    lib = gsb.load_library()
    ctx = gsb.rasterizer._pool(0).take()
    ctx.bind_stream()
    two = torch.full((1,), 2.0, device="cuda")
    scratch = torch.zeros_like(grad)
    dp, dt = _t(pred), _t(tgt)
    dm = None if mask is None else _t(mask)
    assert lib.gs_fused_l1_ssim(ctx.ptr, dp.data_ptr(), dt.data_ptr(),
                                None if dm is None else dm.data_ptr(), W, H, 0.2, 0.7,
                                scratch.data_ptr(), two.data_ptr()) == 0
    torch.cuda.synchronize()
    ctx.release()
    assert abs(float(two) - 2.0 - float(loss)) < 1e-6
    base = torch.ones_like(grad)
    _, acc = gsb.fused_l1_ssim(_t(pred), _t(tgt), None if mask is None else _t(mask), 0.2, 0.7,
                               grad=base)
    assert torch.allclose(acc - 1.0, grad, atol=1e-7)


@pytest.mark.parametrize("masked", [False, True])
def test_ssim_metric_matches_float64_oracle(masked):
    """Large reduction as test_ssim_metric_large_reduction (2e-5), deterministic,
    and an empty mask gives 0."""
    W, H = (191, 137) if masked else (1920, 1276)
    P = W * H
    p = np.arange(P)
    mask = (((p % W + p // W) % 7) == 0).astype(np.float32).reshape(H, W)
    tgt = np.empty((3, P), np.float32)
    pred = np.empty((3, P), np.float32)
    for c in range(3):
        base = 0.15 + 0.7 * ((p * 37 + c * 71) % 1021) / 1021.0
        tgt[c] = base
        pred[c] = np.clip(base + 0.13 * np.sin((p % W) * 0.19 + (p // W) * 0.11 + c), 0, 1)
    tgt = tgt.reshape(3, H, W)
    pred = pred.reshape(3, H, W)
    m = _t(mask) if masked else None
    score = gsb.ssim_metric(_t(pred), _t(tgt), m)
    ref = S.ssim_metric(pred, tgt, mask if masked else None)
    assert abs(score - ref) < 2e-5, (score, ref)
    assert score == gsb.ssim_metric(_t(pred), _t(tgt), m)
    if masked:
        assert gsb.ssim_metric(_t(pred), _t(tgt), torch.zeros_like(m)) == 0.0


def test_rejects_images_of_ten_pixels_or_less():
    x = torch.zeros((3, 10, 40), device="cuda")
    with pytest.raises(Exception, match="width and height > 10"):
        gsb.fused_l1_ssim(x, x)


ref = pytest.importorskip("oracle.reference")


@pytest.mark.skipif(not ref.ssim_available(), reason="reference SSIM kernels not built")
@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("size", [(13, 13), (97, 61), (1920, 1080), (2051, 1027)])
def test_matches_reference_kernels(masked, size):
    """Against the reference's own kernels (photara fused_ssim.cu, built in
    oracle/_ref): the same float32 expressions in the same order, so the
    gradient is bit-identical; the loss differs only in the order of its
    float32 partial sums."""
    W, H = size
    g = torch.Generator(device="cuda").manual_seed(W * 7 + H + masked)
    tgt = torch.rand((3, H, W), device="cuda", generator=g)
    pred = (tgt + 0.1 * torch.randn((3, H, W), device="cuda", generator=g)).clamp(0, 1)
    mask = (torch.rand((H, W), device="cuda", generator=g) > 0.3).float() if masked else None
    base = torch.randn((3, H, W), device="cuda", generator=g)
    lo, go = gsb.fused_l1_ssim(pred, tgt, mask, 0.2, 0.9, grad=base.clone())
    lr, gr = ref.fused_l1_ssim(pred, tgt, mask, 0.2, 0.9, grad=base.clone())
    torch.cuda.synchronize()
    assert torch.equal(go, gr), (go - gr).abs().max().item()
    assert abs(float(lo) - float(lr)) <= 2e-6 * abs(float(lr)) + 1e-9
    mo, mr = gsb.ssim_metric(pred, tgt, mask), ref.ssim_metric(pred, tgt, mask)
    assert abs(mo - mr) <= 1e-6, (mo, mr)
