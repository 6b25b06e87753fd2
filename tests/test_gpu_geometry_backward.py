"""Geometry-channel backward (median depth and normals) against the reference.

The reference differentiates its median-depth and normal outputs
(render_backward.cu:47-151 median_scale_walk, the GEOMETRY branches of
blend_bucket_backward :156-519, the ray-plane / normal chain of
geometry.cuh:617-757). Here the same loss gradients go through both
libraries on the same device inputs; the checker is the reference library
itself (oracle/_ref), driven by ref_backward_geometry.

Tolerance: the activated-space parameter gradients within GEO_REL_L2 relative
L2. Both sides add float32 partials with atomics in different orders, and the
reference restarts each 32-instance bucket from stored snapshots while this
library recovers the transmittance backwards, so agreement is to rounding,
not bit for bit.
"""
import pytest
import torch

from helpers import camera_of, device_model, gsb

ref = pytest.importorskip("oracle.reference")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]

GEO_REL_L2 = 1e-3


def rel_l2(a, b):
    a = a.double().flatten()
    b = b.double().flatten()
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


def _grads(scene_name, seed, depth=True, normal=True, alpha=True):
    if not ref.available():
        pytest.skip("reference library not built (oracle/_ref)")
    scene = gsb.make_scene(scene_name, seed=seed)
    model = device_model(scene)
    cam = camera_of(scene)
    opts = gsb.RasterizeOptions(active_sh_degree=3, require_depth=True, background=(0.1, 0.2, 0.3))
    ours = gsb.Rasterizer().forward(model, cam, opts)
    torch.cuda.synchronize()
    theirs = ref.forward(model, cam, background=(0.1, 0.2, 0.3), need_depth=True)
    assert torch.equal(ours.median_depth, theirs["median_depth"])
    assert (ours.normal - theirs["normal"]).abs().max().item() <= 1e-5
    g = torch.Generator(device="cuda").manual_seed(seed)
    H, W = cam.height, cam.width
    gc = torch.randn((3, H, W), device="cuda", generator=g) * 1e-3
    ga = torch.randn((H, W), device="cuda", generator=g) * 1e-3 if alpha else None
    gd = torch.randn((H, W), device="cuda", generator=g) * 1e-3 if depth else None
    gn = torch.randn((3, H, W), device="cuda", generator=g) * 1e-3 if normal else None
    grads = gsb.Rasterizer().backward(model, ours, gc, ga, grad_depth=gd, grad_normal=gn,
                                      activated_gradients=True)
    z = lambda *s: torch.zeros(s, device="cuda")
    rg = ref.backward_geometry(theirs, gc, ga if alpha else z(H, W),
                               gd if depth else z(H, W), gn if normal else z(3, H, W),
                               model.size(), model.sh.numel(), model.means.device)
    torch.cuda.synchronize()
    pairs = {
        "means": (grads.means, rg["means"]),
        "scales": (grads.log_scales, rg["scales"]),
        "rotations": (grads.quaternions, rg["rotations"]),
        "opacities": (grads.opacity_logits.flatten(), rg["opacities"]),
        "sh": (grads.sh.flatten(), rg["sh"]),
    }
    return {k: rel_l2(a, b) for k, (a, b) in pairs.items()}


@pytest.mark.parametrize("scene_name,seed", [("small", 1), ("g16k_256", 2), ("mid", 3),
                                             ("g1m_1080p", 0)])
def test_geometry_backward_matches_reference(scene_name, seed):
    errs = _grads(scene_name, seed)
    assert all(e < GEO_REL_L2 for e in errs.values()), errs


@pytest.mark.parametrize("depth,normal", [(True, False), (False, True)])
def test_depth_only_and_normal_only_gradients(depth, normal):
    errs = _grads("g16k_256", 5, depth=depth, normal=normal, alpha=False)
    assert all(e < GEO_REL_L2 for e in errs.values()), errs


def test_geometry_gradients_need_a_depth_forward():
    scene = gsb.make_scene("tiny", seed=0)
    model, cam = device_model(scene), camera_of(scene)
    r = gsb.Rasterizer().forward(model, cam, gsb.RasterizeOptions(active_sh_degree=3))
    gd = torch.zeros((cam.height, cam.width), device="cuda")
    with pytest.raises(gsb._lib.StateError):
        gsb.Rasterizer().backward(model, r, torch.zeros_like(r.color), None, grad_depth=gd)


def test_geometry_backward_with_fused_adam_runs_and_matches_unfused():
    """The geometry gradients reach the fused structure Adam: one fused step
    moves the parameters as an Adam step on the unfused gradients does."""
    scene = gsb.make_scene("g16k_256", seed=9)
    cam = camera_of(scene)
    opts = gsb.RasterizeOptions(active_sh_degree=3, require_depth=True)
    g = torch.Generator(device="cuda").manual_seed(9)
    H, W = cam.height, cam.width
    gc = torch.randn((3, H, W), device="cuda", generator=g) * 1e-3
    gd = torch.randn((H, W), device="cuda", generator=g) * 1e-3
    gn = torch.randn((3, H, W), device="cuda", generator=g) * 1e-3
    m1 = device_model(scene)
    r1 = gsb.Rasterizer().forward(m1, cam, opts)
    plain = gsb.Rasterizer().backward(m1, r1, gc, None, grad_depth=gd, grad_normal=gn)
    m2 = device_model(scene)
    z = torch.zeros_like
    st = dict(means_first=z(m2.means), means_second=z(m2.means),
              scales_first=z(m2.log_scales), scales_second=z(m2.log_scales),
              rotations_first=z(m2.quaternions), rotations_second=z(m2.quaternions),
              opacity_first=z(m2.opacity_logits), opacity_second=z(m2.opacity_logits))
    sa = gsb.StructureAdamUpdate(**st, means_lr=1e-3, scales_lr=1e-3, quaternions_lr=1e-3,
                                 opacities_lr=1e-3, correction1=0.1, correction2=0.001)
    r2 = gsb.Rasterizer().forward(m2, cam, opts)
    gsb.Rasterizer().backward(m2, r2, gc, None, grad_depth=gd, grad_normal=gn, structure_adam=sa)
    torch.cuda.synchronize()
    # first moments after one step are (1 - beta1) * gradient
    assert rel_l2(st["means_first"], 0.1 * plain.means) < 1e-5
    assert rel_l2(st["scales_first"], 0.1 * plain.log_scales) < 1e-5
