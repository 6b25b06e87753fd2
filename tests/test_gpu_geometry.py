"""Median-depth and normal channels (render_forward.cu:274-525 with GEOMETRY,
ray plane / normal of geometry.cuh:255-275) against the reference rasterizer
itself (oracle/_ref, need_depth) and the CPU oracle, on seeded scenes.

Bars: median depth and normals within 1e-5 absolute of the reference except
where a probe's decision flips on an ulp (a stated small fraction of pixels);
against the FP32 oracle (different exp / rsqrt / division implementations)
within 1e-3 absolute on the same fraction; colour, alpha and the backward
state identical to the colour-only forward.
"""
import numpy as np
import pytest
import torch

from helpers import camera_of, device_model, gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]

cpu = pytest.importorskip("oracle.cpu")
ref = pytest.importorskip("oracle.reference")


def _ours(scene_name, seed):
    scene = gsb.make_scene(scene_name, seed=seed)
    model = device_model(scene)
    cam = camera_of(scene)
    opts = gsb.RasterizeOptions(active_sh_degree=3, require_depth=True)
    r = gsb.Rasterizer().forward(model, cam, opts)
    torch.cuda.synchronize()
    return scene, model, cam, r


def _close_fraction(a, b, atol):
    return float((np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)) <= atol).mean())


@pytest.mark.parametrize("scene_name,seed", [("small", 1), ("g16k_256", 2), ("mid", 3)])
def test_depth_and_normal_match_reference(scene_name, seed):
    if not ref.available():
        pytest.skip("reference library not built (oracle/_ref)")
    scene, model, cam, ours = _ours(scene_name, seed)
    theirs = ref.forward(model, cam, need_depth=True)
    assert torch.equal(ours.color, theirs["color"]) or \
        float((ours.color - theirs["color"]).abs().max()) <= 1e-5
    d, rd = ours.median_depth.cpu().numpy(), theirs["median_depth"].cpu().numpy()
    nrm, rn = ours.normal.cpu().numpy(), theirs["normal"].cpu().numpy()
    assert np.isfinite(d).all() and np.isfinite(nrm).all()
    assert (d > 0).mean() > 0.3, "too few pixels with a median depth to compare"
    assert _close_fraction(d, rd, 1e-5) >= 0.999, _close_fraction(d, rd, 1e-5)
    assert _close_fraction(nrm, rn, 1e-5) >= 0.999, _close_fraction(nrm, rn, 1e-5)


@pytest.mark.parametrize("scene_name,seed", [("small", 4), ("g16k_256", 5)])
def test_depth_and_normal_match_cpu_oracle(scene_name, seed):
    scene, model, cam, ours = _ours(scene_name, seed)
    o = cpu.render(scene, use_double=False)
    og = cpu.geometry(scene, o)
    d = ours.median_depth.cpu().numpy()
    assert _close_fraction(d, og["median_depth"], 1e-3) >= 0.995
    assert _close_fraction(ours.normal.cpu().numpy(), og["normal"], 1e-3) >= 0.995
    # a pixel has a median depth exactly where its transmittance ends <= 0.45
    alpha = ours.alpha.cpu().numpy()
    assert ((d > 0) <= (alpha >= 0.55 - 1e-6)).all()


def test_geometry_forward_keeps_colour_and_backward():
    scene = gsb.make_scene("g16k_256", seed=6)
    model = device_model(scene)
    cam = camera_of(scene)
    plain = gsb.Rasterizer().forward(model, cam, gsb.RasterizeOptions(active_sh_degree=3))
    geo = gsb.Rasterizer().forward(model, cam, gsb.RasterizeOptions(active_sh_degree=3,
                                                                    require_depth=True))
    assert torch.equal(plain.color, geo.color) and torch.equal(plain.alpha, geo.alpha)
    assert torch.equal(plain.visibility, geo.visibility)
    gc = torch.full_like(plain.color, 1e-3)
    g1 = gsb.Rasterizer().backward(model, plain, gc, torch.zeros_like(plain.alpha))
    g2 = gsb.Rasterizer().backward(model, geo, gc, torch.zeros_like(geo.alpha))
    for k in ("means", "log_scales", "quaternions", "opacity_logits", "sh"):
        a, b = getattr(g1, k), getattr(g2, k)
        assert float((a - b).norm() / b.norm().clamp_min(1e-30)) < 1e-5, k
    # zero median-depth and normal gradients through the geometry-channel
    # adjoint give the colour-only gradients (to float rounding)
    geo2 = gsb.Rasterizer().forward(model, cam, gsb.RasterizeOptions(active_sh_degree=3,
                                                                     require_depth=True))
    g3 = gsb.Rasterizer().backward(model, geo2, gc, torch.zeros_like(geo2.alpha),
                                   grad_depth=torch.zeros_like(geo2.alpha),
                                   grad_normal=torch.zeros_like(geo2.normal))
    for k in ("means", "log_scales", "quaternions", "opacity_logits", "sh"):
        a, b = getattr(g3, k), getattr(g1, k)
        assert float((a - b).norm() / b.norm().clamp_min(1e-30)) < 1e-5, k
