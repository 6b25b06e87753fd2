"""CPU tests: the oracle pinned to the reference (golden fixtures made by the
reference library, known-answer cases of the reference's own tests, finite
differences), the SH Adam codec, the C-ABI export list and host-side checks.
No GPU needed.
"""
import re
from pathlib import Path

import numpy as np
import pytest

from helpers import gsb
from oracle import cpu

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _golden_cases():
    return sorted(GOLDEN.glob("ref_*.npz"))


@pytest.mark.parametrize("path", _golden_cases(), ids=lambda p: p.stem)
def test_oracle_matches_reference_golden(path):
    """Oracle vs outputs of the reference rasterizer on the same seeded scene.

    Bars: radii, visibility, tile ranges and the sorted draw list identical
    (on these fixtures they are; libm vs fast-math transcendental ulps could in
    principle move a tile-boundary decision, which would show up here);
    images within 1e-5; gradients within 2e-5 relative L2 (measured: images
    <= 3.4e-6, gradients <= 2.2e-6).
    """
    from tests.golden.make_golden import loss_grads
    m = re.match(r"ref_(\w+)_s(\d+)", path.stem)
    name, seed = m.group(1), int(m.group(2))
    ref = np.load(path)
    scene = gsb.make_scene(name, seed=seed)
    bg = tuple(ref["background"].tolist())
    o = cpu.render(scene, background=bg)
    assert np.array_equal(o["radii"], ref["radii"])
    assert np.array_equal(o["visibility"], ref["visibility"])
    assert o["instances"] == int(ref["instances"]) and o["visible"] == int(ref["visible"])
    assert np.array_equal(o["ranges"].astype(np.int64), ref["ranges"].astype(np.int64))
    assert np.array_equal(o["values"], ref["values"].astype(np.uint32))
    assert np.abs(o["color"] - ref["color"]).max() <= 1e-5
    assert np.abs(o["alpha"] - ref["alpha"]).max() <= 1e-5
    gc, ga = loss_grads(scene, seed)
    g = cpu.backward(scene, o, gc, ga, activated=True)
    for key, ours in (("means", g["means"]), ("scales", g["scales"]),
                      ("rotations", g["rotations"]), ("opacities", g["opacities"]),
                      ("refine_weight", g["refine_weight"])):
        assert rel_l2(ours, ref["grad_" + key]) <= 2e-5, key
    if "grad_sh" in ref:
        assert rel_l2(g["sh"].ravel(), ref["grad_sh"]) <= 2e-5


def _single_scene(mean=(0.5, 0.0, 2.0)):
    s = gsb.make_scene("tiny", seed=0, count=1)
    s.means[:] = np.asarray([mean], np.float32)
    s.log_scales[:] = np.log(0.15)
    s.quaternions[:] = np.asarray([[1.0, 0, 0, 0]], np.float32)
    s.opacity_logits[:] = 2.0
    s.sh[:] = 0.0
    s.sh[0, 0] = [0.5, 0.25, 0.1]
    s.width, s.height, s.fx, s.fy, s.cx, s.cy = 48, 32, 40.0, 40.0, 23.5, 15.5
    return s


def test_oracle_single_gaussian_known_answers():
    """Background blend identity and colour gradient = sum of alpha
    (photara/tests/splat_test.cpp:2369-2460, :881-946)."""
    s = _single_scene()
    black = cpu.render(s, sh_degree=0)
    assert black["instances"] > 0 and black["visibility"].tolist() == [1.0]
    bg = (0.1, 0.3, 0.7)
    col = cpu.render(s, background=bg, sh_degree=0)
    diff = col["color"] - black["color"] - (1 - black["alpha"])[None] * np.asarray(bg)[:, None, None]
    assert np.abs(diff).max() < 5e-6
    # d(sum of red)/d(red colour) of a lone splat = sum of alpha
    gc = np.zeros((3, s.height, s.width), np.float32)
    gc[0] = 1.0
    g = cpu.backward(s, black, gc, sh_degree=0)
    assert abs(g["grad12"][0, 8] - black["alpha"].sum()) < 2e-6 * max(black["alpha"].sum(), 1)
    # closed form of the DC colour: 0.5 + SH0 * coefficient
    expected_rgb = 0.5 + 0.28209479177387814 * np.asarray([0.5, 0.25, 0.1])
    assert np.allclose(black["rgb"][0], expected_rgb, atol=1e-6)


def test_oracle_fp32_and_fp64_compositing_agree():
    s = gsb.make_scene("small", seed=3)
    a = cpu.render(s, use_double=True)
    b = cpu.render(s, use_double=False)
    assert np.abs(a["color"] - b["color"]).max() < 5e-6
    assert np.array_equal(a["last"], b["last"])


def _fd_scene():
    """Three overlapping anisotropic Gaussians, large in pixels (sigma ~5-10 px),
    so the alpha >= 1/255 cut-off ring (a discontinuity the analytic adjoint
    ignores, as the reference's does) is a small share of each gradient."""
    s = gsb.make_scene("tiny", seed=0, count=3)
    s.width, s.height, s.fx, s.fy, s.cx, s.cy = 64, 48, 64.0, 64.0, 32.0, 24.0
    s.means[:] = np.asarray([[-0.2, 0.1, 3.0], [0.25, -0.05, 3.4], [0.0, 0.3, 3.8]], np.float32)
    s.log_scales[:] = np.log(np.asarray([[0.35, 0.2, 0.3], [0.25, 0.4, 0.2],
                                         [0.3, 0.3, 0.15]], np.float32))
    q = np.asarray([[0.9, 0.2, -0.3, 0.1], [0.7, -0.4, 0.2, 0.5], [0.95, 0.1, 0.1, -0.2]])
    s.quaternions[:] = (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)
    s.opacity_logits[:] = np.asarray([[0.5], [1.2], [-0.3]], np.float32)
    return s


def test_oracle_gradients_match_finite_differences():
    """Central differences of the oracle's own FP64-composited forward (FD
    pattern of photara/tests/splat_test.cpp:948-1039) on every raw parameter
    of three Gaussians. Smooth loss weights; tolerance 1% of the largest
    gradient of the parameter group + 3% of |fd|."""
    s = _fd_scene()
    yy, xx = np.mgrid[0:s.height, 0:s.width].astype(np.float32)
    w = np.stack([1.0 + 0.5 * np.sin(xx / 9.0), 0.8 + 0.4 * np.cos(yy / 7.0),
                  0.6 + 0.3 * np.sin((xx + yy) / 11.0)]).astype(np.float32)
    u = (0.3 * np.cos(xx / 13.0) * np.sin(yy / 10.0)).astype(np.float32)

    def loss(scene):
        f = cpu.render(scene)
        return float((f["color"] * w).sum() + (f["alpha"] * u).sum())

    f0 = cpu.render(s)
    g = cpu.backward(s, f0, w, u)
    groups = {"means": (s.means, g["means"]), "log_scales": (s.log_scales, g["scales"]),
              "quaternions": (s.quaternions, g["rotations"]),
              "opacity_logits": (s.opacity_logits, g["opacities"].reshape(-1, 1)),
              "sh": (s.sh, g["sh"])}
    h = 2e-4
    for name, (arr, grad) in groups.items():
        gmax = np.abs(grad).max()
        idxs = list(np.ndindex(arr.shape))
        if name == "sh":
            idxs = [(i, k, c) for i in range(3) for k in (0, 1, 5, 12) for c in (0, 2)]
        for idx in idxs:
            old = arr[idx]
            arr[idx] = old + h
            lp = loss(s)
            arr[idx] = old - h
            lm = loss(s)
            arr[idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(grad[idx] - fd) <= 0.01 * gmax + 0.03 * abs(fd), (name, idx, grad[idx], fd)


def test_half_conversion_matches_numpy():
    """The oracle's fp16 codec helpers round like IEEE binary16 (numpy)."""
    vals = np.concatenate([np.random.default_rng(0).normal(size=2000).astype(np.float32) * s
                           for s in (1e-6, 1e-3, 1.0, 1e3)]).astype(np.float32)
    vals = np.concatenate([vals, np.asarray([0.0, -0.0, 65504.0, 7e-8, 6e-5, 1.0], np.float32)])
    vals = vals[: vals.size // 48 * 48].reshape(-1, 48)
    rows = vals.shape[0]
    # Round trip through the codec's encode of an inactive column: first is
    # re-encoded from its decoded value, so encode(decode(x)) must be x.
    ref_bits = vals.astype(np.float16).view(np.uint16)
    first = ref_bits.copy()
    packed = np.zeros((rows, 48), np.uint8)
    bounds = np.zeros((rows, 4), np.float32)
    param = np.zeros((rows, 48), np.float32)
    grad = np.zeros((rows, 48), np.float32)
    # c1=c2=1 with beta=0.5 gives previous corrections of 1: a stored u decodes
    # to u*(0+eps)*1 and re-encodes to the same u when eps=1 and v=0.
    cpu.sh_adam_rows(param, grad, first, packed, bounds, active=0, lr=0, rest_lr=0, b1=0.5,
                     b2=0.5, c1=1.0, c2=1.0, eps=1.0)
    assert np.array_equal(first, ref_bits)


def test_sh_adam_oracle_first_step():
    """First quantized-Adam step from zero state: the update is -lr*sign(g)
    (bias-corrected Adam), codes span [0, 255] per group."""
    rng = np.random.default_rng(1)
    rows, stride = 64, 48
    param = rng.normal(size=(rows, stride)).astype(np.float32)
    p0 = param.copy()
    grad = rng.normal(size=(rows, stride)).astype(np.float32)
    first = np.zeros((rows, stride), np.uint16)
    packed = np.zeros((rows, stride), np.uint8)
    bounds = np.zeros((rows, 4), np.float32)
    cpu.sh_adam_rows(param, grad, first, packed, bounds, active=48, lr=1e-2, rest_lr=1e-3,
                     b1=0.9, b2=0.999, c1=0.1, c2=0.001, eps=1e-8)
    step = p0 - param
    assert np.allclose(step[:, :3], 1e-2 * np.sign(grad[:, :3]), rtol=1e-3)
    assert np.allclose(step[:, 3:], 1e-3 * np.sign(grad[:, 3:]), rtol=1e-3)
    assert (packed[:, 3:].max(axis=1) == 255).all() and (packed[:, 3:].min(axis=1) == 0).all()
    assert (bounds[:, 0] <= bounds[:, 1]).all() and (bounds[:, 2] <= bounds[:, 3]).all()


def test_c_abi_exports_every_declared_symbol():
    header = (ROOT / "include" / "gsplat_b200.h").read_text()
    declared = re.findall(r"^GS_API\s+[\w\s\*]+?\b(gs_\w+)\(", header, flags=re.M)
    assert len(declared) >= 12
    lib = gsb.load_library()
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) <= set(gsb._lib.SIGNATURES)
    assert lib.gs_abi_version() == 3


def test_host_validation_rejects_cpu_tensors():
    import torch
    s = gsb.make_scene("tiny", seed=0)
    t = lambda a: torch.from_numpy(a)
    model = gsb.GaussianModel(t(s.means), t(s.log_scales), t(s.quaternions),
                              t(s.opacity_logits), t(s.sh), 3)
    cam = gsb.Camera(s.world_to_camera, s.position, s.fx, s.fy, s.cx, s.cy, s.width, s.height)
    with pytest.raises(ValueError, match="contiguous CUDA"):
        gsb.Rasterizer().forward(model, cam)


def test_oracle_median_depth_single_gaussian_known_answer():
    """One opaque Gaussian facing the camera: along the central ray the
    transmittance is sqrt(1 - alpha g(t)) in front of the peak (the probe
    formula of render_forward.cu:468-480), so it crosses 0.5 where
    alpha g = 0.75: at t_peak - sigma sqrt(2 ln(alpha / 0.75)); the median
    depth is that distance times the ray's z (1 on the optical axis)."""
    import types
    z, s = 3.0, 0.05
    sc = types.SimpleNamespace(
        count=1, width=64, height=64, fx=64.0, fy=64.0, cx=32.0, cy=32.0,
        world_to_camera=[1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0],
        position=[0.0, 0.0, 0.0],
        means=np.array([[0.0, 0.0, z]], np.float32),
        log_scales=np.full((1, 3), np.log(s), np.float32),
        quaternions=np.array([[1.0, 0, 0, 0]], np.float32),
        opacity_logits=np.array([[6.0]], np.float32),
        sh=np.zeros((1, 16, 3), np.float32))
    f = cpu.render(sc, use_double=False)
    g = cpu.geometry(sc, f)
    a = min(0.99, float(f["conic"][0, 3]))
    expect = z - s * np.sqrt(2.0 * np.log(a / 0.75))
    assert abs(float(g["median_depth"][32, 32]) - expect) <= 2e-4 * z
    assert np.allclose(g["normal"][:, 32, 32], [0.0, 0.0, -1.0], atol=1e-5)
    assert float(g["plane"][0, 3]) == pytest.approx(1.0 / s, rel=1e-5)


def test_ssim_oracle_gradient_matches_central_differences():
    """oracle/ssim_ref.py: the analytic gradient of the fused L1 + SSIM loss
    against central differences (float64), with and without a mask."""
    from oracle import ssim_ref as S
    rng = np.random.default_rng(3)
    H, W = 17, 19
    tgt = rng.uniform(0.1, 0.9, (3, H, W))
    pred = np.clip(tgt + rng.normal(0, 0.1, tgt.shape), 0, 1)
    for mask in (None, (rng.uniform(size=(H, W)) > 0.2).astype(np.float64)):
        _, g, _ = S.fused_l1_ssim(pred, tgt, mask, 0.2, 1.0)
        for (c, y, x) in [(0, 8, 9), (1, 5, 5), (2, 12, 3), (0, 0, 0)]:
            e = 1e-6
            pp, pm = pred.copy(), pred.copy()
            pp[c, y, x] += e
            pm[c, y, x] -= e
            fd = (S.fused_l1_ssim(pp, tgt, mask, 0.2, 1.0)[0] -
                  S.fused_l1_ssim(pm, tgt, mask, 0.2, 1.0)[0]) / (2 * e)
            assert abs(fd - g[c, y, x]) <= 1e-6 + 1e-4 * abs(fd), (c, y, x, fd, g[c, y, x])


def test_ssim_oracle_constant_images_known_answer():
    from oracle import ssim_ref as S
    p, r = 0.25, 0.75
    loss, _, ssim = S.fused_l1_ssim(np.full((3, 40, 50), p), np.full((3, 40, 50), r), None)
    expect = (2 * p * r + 1e-4) / (p * p + r * r + 1e-4)
    # the float32 window values sum to 1 - 3.1e-8 exactly, which leaves a
    # variance of about 6e-8 p^2 on a constant image: 1.7e-5 of SSIM
    assert np.abs(ssim[:, 5:35, 5:45] - expect).max() < 3e-5
    assert abs(loss - (0.8 * (r - p) + 0.2 * (1 - expect))) < 3e-5


def _loss_case(rng, H=14, W=17):
    from oracle import loss_ref
    yy, xx = np.mgrid[0:H, 0:W]
    depth = 2.0 + 0.05 * xx + 0.03 * yy + 0.02 * rng.normal(size=(H, W))
    normal = rng.normal(size=(3, H, W))
    normal /= np.linalg.norm(normal, axis=0)
    return loss_ref, depth, normal


def test_depth_normal_consistency_gradient_matches_central_differences():
    """oracle/loss_ref.py: the analytic gradients of the depth-normal
    consistency term (cuda_ops.cu:999-1071) against central differences of
    its loss, with respect to depth and to the rendered normal."""
    rng = np.random.default_rng(5)
    loss_ref, depth, normal = _loss_case(rng)
    intr = (20.0, 22.0, 8.3, 6.9)
    _, gd, gn = loss_ref.depth_normal_consistency(depth, normal, *intr, 0.5)
    e = 1e-6
    for (y, x) in [(0, 5), (3, 4), (7, 8), (13, 16), (6, 0)]:
        dp, dm = depth.copy(), depth.copy()
        dp[y, x] += e
        dm[y, x] -= e
        fd = (loss_ref.depth_normal_consistency(dp, normal, *intr, 0.5)[0] -
              loss_ref.depth_normal_consistency(dm, normal, *intr, 0.5)[0]) / (2 * e)
        assert abs(fd - gd[y, x]) <= 1e-7 + 1e-5 * abs(fd), (y, x, fd, gd[y, x])
    for (c, y, x) in [(0, 3, 4), (2, 7, 8), (1, 12, 15)]:
        npl, nmi = normal.copy(), normal.copy()
        npl[c, y, x] += e
        nmi[c, y, x] -= e
        fd = (loss_ref.depth_normal_consistency(depth, npl, *intr, 0.5)[0] -
              loss_ref.depth_normal_consistency(depth, nmi, *intr, 0.5)[0]) / (2 * e)
        assert abs(fd - gn[c, y, x]) <= 1e-9 + 1e-6 * abs(fd)


def test_training_loss_terms_match_their_gradients():
    """oracle/loss_ref.py: each per-pixel term's gradient is the derivative of
    its own scalar (depth robust term, normal prior, alpha BCE, small-image L1)."""
    rng = np.random.default_rng(6)
    loss_ref, depth, normal = _loss_case(rng, 9, 8)  # 8 wide: plain L1 colour term
    H, W = depth.shape
    color = rng.uniform(0, 1, (3, H, W))
    target = rng.uniform(0, 1, (3, H, W))
    tdepth = np.where(rng.uniform(size=(H, W)) > 0.2, depth + 0.1 * rng.normal(size=(H, W)), 0)
    tnormal = rng.normal(size=(3, H, W))
    alpha = rng.uniform(0.05, 0.95, (H, W))
    mask = (rng.uniform(size=(H, W)) > 0.3).astype(np.float64)
    kw = dict(alpha=alpha, median_depth=depth, normal=normal, target_depth=tdepth,
              target_normal=tnormal, mask=mask, photometric_weight=0.7, depth_weight=0.4,
              normal_weight=0.3, match_alpha_weight=0.25, alpha_mode="transparent",
              need_geometry_gradients=True)
    out = loss_ref.training_loss(color, target, **kw)
    e = 1e-6

    def total(**over):
        args = dict(kw)
        args.update(over)
        c = args.pop("color", color)
        return float(loss_ref.training_loss(c, target, **args)["terms"].sum())

    for (y, x) in [(2, 3), (5, 6)]:
        for name, arr, g in (("median_depth", depth, out["depth"]),
                             ("alpha", alpha, out["alpha"])):
            p, m = arr.copy(), arr.copy()
            p[y, x] += e
            m[y, x] -= e
            fd = (total(**{name: p}) - total(**{name: m})) / (2 * e)
            assert abs(fd - g[y, x]) <= 1e-7 + 1e-5 * abs(fd), (name, y, x, fd, g[y, x])
        for c in range(3):
            p, m = normal.copy(), normal.copy()
            p[c, y, x] += e
            m[c, y, x] -= e
            fd = (total(normal=p) - total(normal=m)) / (2 * e)
            assert abs(fd - out["normal"][c, y, x]) <= 1e-7 + 1e-5 * abs(fd)
            p, m = color.copy(), color.copy()
            p[c, y, x] += e
            m[c, y, x] -= e
            fd = (total(color=p) - total(color=m)) / (2 * e)
            assert abs(fd - out["color"][c, y, x]) <= 1e-7 + 1e-5 * abs(fd)


def _split_case(rng, n=64, m=40):
    from oracle import densify_apply_ref as D
    q = rng.normal(size=(n, 4))
    parent = dict(means=rng.normal(size=(n, 3)), log_scales=rng.normal(-3, 0.7, (n, 3)),
                  opacity_logits=rng.normal(0, 1.5, n), quaternions=q)
    parents = rng.choice(n, m, replace=False)
    child = {k: v[parents].copy() for k, v in parent.items()}
    return D, parent, child, parents


def _cov(means, log_scales, q):
    from oracle import densify_apply_ref as D
    qn = q / np.linalg.norm(q, axis=1, keepdims=True)
    R = np.stack([D.rotate(qn, np.tile(e, (len(q), 1))) for e in np.eye(3)], axis=2)
    S = np.exp(log_scales)
    return np.einsum("nij,nj,nkj->nik", R, S * S, R)


def test_split_modes_known_answers():
    """oracle/densify_apply_ref.py against the properties the reference states for
    each split mode (ops.hpp:282-310, cuda_ops.cu:1720-1845)."""
    rng = np.random.default_rng(8)
    D, parent, child, parents = _split_case(rng)
    q = parent["quaternions"][parents]
    cov0 = _cov(parent["means"][parents], parent["log_scales"][parents], q)
    a0 = 1 / (1 + np.exp(-parent["opacity_logits"][parents]))
    # adc_covariance: the two-child mixture keeps the parent's covariance and mean
    P, Cc = D.split(parent, child, parents, "adc_covariance")
    mu_p, mu_c = P["means"][parents], Cc["means"]
    mix = 0.5 * (_cov(mu_p, P["log_scales"][parents], q) + _cov(mu_c, Cc["log_scales"], q))
    d = 0.5 * (mu_c - mu_p)
    mix += np.einsum("ni,nj->nij", d, d)
    assert np.allclose(mix, cov0, rtol=1e-9, atol=1e-15)
    assert np.allclose(0.5 * (mu_p + mu_c), parent["means"][parents], atol=1e-12)
    a1 = 1 / (1 + np.exp(-Cc["opacity_logits"]))
    assert np.allclose(np.clip(1 - (1 - a0) ** (1 / np.sqrt(2)), 1e-6, 1 - 1e-6), a1)
    # igs_random: two children composite back to the parent's alpha
    rs = rng.normal(size=(len(parents), 3))
    P, Cc = D.split(parent, child, parents, "igs_random", random_samples=rs)
    a1 = 1 / (1 + np.exp(-Cc["opacity_logits"]))
    assert np.allclose(1 - (1 - a1) ** 2, a0, atol=1e-9)
    assert np.allclose(P["means"][parents] + Cc["means"], 2 * parent["means"][parents])
    # long_axis: a' = k / (1 + exp(-l) - k); major axis halves, others x0.85
    P, Cc = D.split(parent, child, parents, "long_axis", split_opacity_k=0.6)
    a1 = 1 / (1 + np.exp(-Cc["opacity_logits"]))
    expect = np.clip(0.6 / (1 + np.exp(-parent["opacity_logits"][parents]) - 0.6), 1e-6,
                     1 - 1e-6)
    assert np.allclose(a1, expect)
    ratio = np.exp(Cc["log_scales"] - parent["log_scales"][parents])
    assert np.allclose(np.sort(ratio, axis=1)[:, 1:], 0.85) and np.allclose(ratio.min(1), 0.5)
    # dense_tangent: local z (the normal axis) keeps its scale and offset 0
    P, Cc = D.split(parent, child, parents, "dense_tangent", random_samples=rs)
    assert np.allclose(Cc["log_scales"][:, 2], parent["log_scales"][parents][:, 2])
    # ADC decay
    ls, lo = D.adc_decay(parent["log_scales"], parent["opacity_logits"], 0.01, 0.02)
    assert np.allclose(ls - parent["log_scales"], np.log(0.98))
    assert np.allclose(1 / (1 + np.exp(-lo)),
                       np.clip(1 / (1 + np.exp(-parent["opacity_logits"])) - 0.01, 1e-12,
                               1 - 1e-12))


def test_pruning_score_derivative_is_the_composite_sensitivity():
    """oracle/prune_ref.py: the per-pixel derivative the Speedy-Splat score
    squares (rasterizer.cu:93-146) equals opacity x d(composited colour sum) /
    d(alpha_i) with the other alphas fixed (central differences of the
    front-to-back composite over the entries, background included)."""
    from oracle import prune_ref
    rng = np.random.default_rng(12)
    k = 7
    mean2d = np.zeros((k, 2), np.float32)
    conic = np.zeros((k, 4), np.float32)
    conic[:, 0] = conic[:, 2] = 1e-3
    conic[:, 3] = rng.uniform(0.2, 0.9, k)
    rgb = rng.uniform(0, 1, (k, 4)).astype(np.float32)
    bg = np.array([0.3, 0.1, 0.6])
    px = py = 0.0
    alphas = np.array([min(0.99, c[3] * np.exp(-0.5e-3 * 0)) for c in conic], np.float64)

    def composite(al):
        T, col = 1.0, np.zeros(3)
        for i in range(k):
            col += T * al[i] * rgb[i, :3]
            T *= 1 - al[i]
        return col + T * bg

    image = composite(alphas)
    terms = prune_ref.pixel_terms(np.arange(k), px, py, mean2d, conic, rgb, image, 0.99)
    assert len(terms) == k
    e = 1e-7
    for g, d, per in terms:
        ap, am = alphas.copy(), alphas.copy()
        ap[g] += e
        am[g] -= e
        fd = (composite(ap) - composite(am)) / (2 * e)
        assert abs(d - conic[g, 3] * fd.sum()) <= 1e-6 * (1 + abs(d))
        assert np.allclose(per, alphas[g] * fd, atol=1e-7)
