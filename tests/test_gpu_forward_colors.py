"""Colour reuse (splat_drender Rasterizer::forward_colors,
third_party/splat_drender/src/pipeline.cu:617-649): blending new precomputed
colours over a training forward's draw list gives exactly the render of a
fresh forward with those colours (alpha, termination and draw order do not
depend on the colours), and its gradients to rounding (atomic order)."""
import pytest
import torch

from helpers import camera_of, device_model, gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]


@pytest.mark.parametrize("scene_name,seed", [("small", 0), ("g16k_256", 2)])
def test_reuse_equals_fresh_forward_and_backward(scene_name, seed):
    scene = gsb.make_scene(scene_name, seed=seed)
    model = device_model(scene)
    cam = camera_of(scene)
    n = model.size()
    g = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.rand((n, 3), device="cuda", generator=g)
    b = torch.rand((n, 3), device="cuda", generator=g)
    rast = gsb.Rasterizer()
    bg = (0.2, 0.1, 0.4)
    first = rast.forward(model, cam, gsb.RasterizeOptions(colors_precomp=a, background=bg))
    reused = rast.forward_colors(first, b)
    fresh = rast.forward(model, cam, gsb.RasterizeOptions(colors_precomp=b, background=bg))
    torch.cuda.synchronize()
    assert first.context is None
    assert torch.equal(reused.color, fresh.color)
    assert torch.equal(reused.alpha, fresh.alpha)
    assert torch.equal(reused.visibility, fresh.visibility)
    assert not torch.equal(reused.color, first.color)
    dl = torch.randn(fresh.color.shape, device="cuda", generator=g) * 1e-3
    g1 = rast.backward(model, reused, dl, None)
    g2 = rast.backward(model, fresh, dl, None)
    # per-Gaussian gradients are summed over warps and tiles with float atomics
    # in an unspecified order, so two backward passes agree to rounding only
    # (small frames composite with one pixel per thread: eight warp partial
    # sums per Gaussian and tile, so cancellation leaves up to ~2e-5 of the
    # largest gradient); a wrong draw list or colour slot would differ at O(1)
    for name in ("means", "log_scales", "quaternions", "opacity_logits", "colors_precomp"):
        x, y = getattr(g1, name), getattr(g2, name)
        scale = y.abs().max().item() + 1e-30
        assert (x - y).abs().max().item() <= 1e-4 * scale, name


def test_reuse_needs_a_training_forward_with_precomputed_colours():
    scene = gsb.make_scene("small", seed=1)
    model = device_model(scene)
    cam = camera_of(scene)
    rast = gsb.Rasterizer()
    colors = torch.rand((model.size(), 3), device="cuda")
    with pytest.raises(Exception, match="precomputed colors"):
        rast.forward_colors(rast.forward(model, cam), colors)
    with pytest.raises(Exception, match="training forward"):
        rast.forward_colors(rast.forward(model, cam, gsb.RasterizeOptions(
            colors_precomp=colors, record_backward_state=False)), colors)
    # the C ABI refuses an SH forward too
    r = rast.forward(model, cam)
    lib = gsb.load_library()
    out = gsb._lib.Outputs(r.color.data_ptr(), r.alpha.data_ptr(), None, None, None, None)
    import ctypes
    assert lib.gs_forward_colors(r.context.ctx.ptr, colors.data_ptr(), ctypes.byref(out)) != 0
