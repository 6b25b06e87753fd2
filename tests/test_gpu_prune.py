"""Speedy-Splat pruning scores (photara CudaRasterizer::pruning_scores,
rasterizer.cu:450-490, kernel :93-146) on the library's kernel, against the
reference's own kernel (oracle/_ref/libprune_ref.so over the reference
rasterizer's forward: 1e-5 relative, both sum float32 values with atomics in
an unspecified order) and the float64 restatement (oracle/prune_ref.py)
over the CPU oracle's forward, whose draw list is identical to this
library's.

Bars: relative L2 error of the score vector 1e-4 and every score within
2e-3 of the largest (float32 residuals subtract the blended colour from the
rendered image, float64 in the restatement); Gaussians never blended score
exactly 0; scores add over calls; a forward that did not record its
per-pixel state is refused."""
import numpy as np
import pytest
import torch

from helpers import camera_of, device_model, gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]

cpu = pytest.importorskip("oracle.cpu")
prune_ref = pytest.importorskip("oracle.prune_ref")
ref = pytest.importorskip("oracle.reference")


@pytest.mark.parametrize("gaussian_pop", [False, True])
@pytest.mark.parametrize("scene_name,seed", [("small", 0), ("small", 3), ("g16k_256", 1)])
def test_scores_match_float64_restatement(scene_name, seed, gaussian_pop):
    scene = gsb.make_scene(scene_name, seed=seed)
    model = device_model(scene)
    cam = camera_of(scene)
    bg = (0.1, 0.2, 0.3)
    opts = gsb.RasterizeOptions(active_sh_degree=3, background=bg)
    ours = gsb.Rasterizer().pruning_scores(model, cam, opts, gaussian_pop=gaussian_pop)
    torch.cuda.synchronize()
    fwd = cpu.render(scene, background=bg)
    exp = prune_ref.pruning_scores(fwd, scene.width, scene.height, model.size(),
                                   gaussian_pop=gaussian_pop)
    got = ours.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(got - exp) <= 1e-4 * np.linalg.norm(exp)
    assert np.abs(got - exp).max() <= 2e-3 * np.abs(exp).max()
    assert np.all(got[exp == 0] == 0)
    assert (exp > 0).sum() > 0.5 * model.size()


def test_scores_add_over_calls_and_need_recorded_state():
    scene = gsb.make_scene("small", seed=5)
    model = device_model(scene)
    cam = camera_of(scene)
    rast = gsb.Rasterizer()
    a = rast.pruning_scores(model, cam)
    b = rast.pruning_scores(model, cam)
    assert torch.equal(a, b) or torch.allclose(a, b, rtol=1e-5, atol=0)
    # the C ABI adds into the caller's scores and refuses an inference-only render
    lib = gsb.load_library()
    r = rast.forward(model, cam, gsb.RasterizeOptions(record_backward_state=False))
    live = r.context
    live.ctx.bind_stream()
    acc = torch.zeros_like(a)
    rc = lib.gs_pruning_scores(live.ctx.ptr, r.color.data_ptr(), 0, acc.data_ptr())
    assert rc != 0 and b"record_backward_state" in lib.gs_last_error(live.ctx.ptr)
    r = rast.forward(model, cam)
    live = r.context
    live.ctx.bind_stream()
    acc = a.clone()
    assert lib.gs_pruning_scores(live.ctx.ptr, r.color.data_ptr(), 0, acc.data_ptr()) == 0
    torch.cuda.synchronize()
    assert torch.allclose(acc, 2 * a, rtol=1e-5, atol=0)


@pytest.mark.skipif(not ref.prune_available(), reason="reference score kernel not built")
@pytest.mark.parametrize("gaussian_pop", [False, True])
@pytest.mark.parametrize("scene_name,seed", [("small", 0), ("g16k_256", 1), ("mid", 2)])
def test_scores_match_reference_kernel(scene_name, seed, gaussian_pop):
    scene = gsb.make_scene(scene_name, seed=seed)
    model = device_model(scene)
    cam = camera_of(scene)
    bg = (0.1, 0.2, 0.3)
    ours = gsb.Rasterizer().pruning_scores(model, cam, gsb.RasterizeOptions(
        active_sh_degree=3, background=bg), gaussian_pop=gaussian_pop)
    theirs, _ = ref.pruning_scores(model, cam, background=bg, gaussian_pop=gaussian_pop)
    torch.cuda.synchronize()
    scale = theirs.abs().max().item()
    assert scale > 0
    assert (ours - theirs).abs().max().item() <= 1e-5 * scale
    assert torch.equal(ours == 0, theirs == 0)
