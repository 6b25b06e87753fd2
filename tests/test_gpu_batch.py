"""Batched multi-view rendering (gs_batch_*) against the single-view path.

Per view, the batched images must equal Rasterizer.forward on that camera:
the per-pixel blend sequence does not depend on the tile shape or the tile
schedule (a pixel only blends Gaussians whose alpha >= 1/255 contour covers
it, and the tile walk covers that contour exactly). Tolerances stated here:
  * colour / alpha: at most 1e-6 absolute and identical on >= 99.9% of pixels;
  * radii identical;
  * gradients (summed over views): relative L2 <= 2e-5 against the sum of the
    single-view backward passes (float atomics accumulate in another order).
"""
import importlib

import numpy as np
import pytest
import torch

from helpers import gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]

batch = importlib.import_module("photara-studio_b200.batch")
scenes = importlib.import_module("photara-studio_b200.scenes")

SIZES = ((160, 120), (128, 72), (200, 150), (96, 96), (64, 48), (72, 40))


def rel_l2(a, b):
    a = a.double().flatten()
    b = b.double().flatten()
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


def _setup(n=20000, views=5, seed=3):
    arrays, ring = scenes.make_ring_batch(n, views=views, sizes=SIZES, radius=6.0, half=2.0,
                                          seed=seed)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    model = gsb.GaussianModel(t(arrays.means), t(arrays.log_scales), t(arrays.quaternions),
                              t(arrays.opacity_logits), t(arrays.sh), 3)
    cams = [gsb.look_at_camera(v.eye, (0, 0, 0), (0, 1, 0), v.width, v.height, v.focal)
            for v in ring]
    return model, cams


def _single(model, cams, grads_in=None):
    rast = gsb.Rasterizer()
    opts = gsb.RasterizeOptions(active_sh_degree=3)
    outs, total = [], None
    for k, c in enumerate(cams):
        r = rast.forward(model, c, opts)
        outs.append((r.color.clone(), r.alpha.clone(), r.radii.clone()))
        if grads_in is not None:
            g = rast.backward(model, r, grads_in[k].contiguous(), None)
            parts = [g.means, g.log_scales, g.quaternions, g.opacity_logits.flatten(), g.sh]
            total = parts if total is None else [a + b for a, b in zip(total, parts)]
    return outs, total


def _grad_views(res, seed=0):
    g = torch.Generator("cuda").manual_seed(seed)
    flat = torch.randn(res.color.numel(), device="cuda", generator=g) * 1e-3
    per_view = []
    for v, (w, h, off) in enumerate(res.views):
        per_view.append(flat[3 * off:3 * (off + w * h)].view(3, h, w))
    return flat, per_view


SHAPES = [(8, 8, 1, "dynamic"), (8, 8, 2, "static"), (16, 16, 2, "heavy_first"),
          (16, 16, 4, "dynamic"), (16, 16, 4, "static"), (16, 16, 4, "heavy_first"),
          (16, 32, 2, "dynamic"), (16, 32, 4, "heavy_first")]


@pytest.mark.parametrize("tw,th,ppt,sched", SHAPES)
def test_batch_matches_single_view(tw, th, ppt, sched):
    model, cams = _setup()
    br = batch.BatchRasterizer()
    br.plan(model, cams, gsb.RasterizeOptions(active_sh_degree=3),
            batch.BatchSchedule(tw, th, ppt, sched))
    res = br.forward()
    flat, per_view = _grad_views(res)
    grads = br.backward(flat)
    torch.cuda.synchronize()
    info = br.info()
    assert info["overflow"] == 0 and info["device_error"] == 0 and info["instances"] > 0
    single, total = _single(model, cams, per_view)
    for v, (c, a, rad) in enumerate(single):
        bc, ba = res.view_color(v), res.view_alpha(v)
        assert float((bc - c).abs().max()) <= 1e-6
        assert float((ba - a).abs().max()) <= 1e-6
        assert float((bc == c).float().mean()) >= 0.999
        # radii agree wherever both tile grids keep the Gaussian; one whose
        # footprint only reaches the padded border of one grid is culled by the
        # other (it reaches no pixel either way)
        both = (res.radii[v] > 0) & (rad > 0)
        assert torch.equal(res.radii[v][both], rad[both])
        if (tw, th) == (16, 16):
            assert torch.equal(res.radii[v], rad)
    got = [grads.means, grads.log_scales, grads.quaternions, grads.opacity_logits.flatten(),
           grads.sh]
    for name, a, b in zip(("means", "log_scales", "quaternions", "opacity", "sh"), got, total):
        assert rel_l2(a, b) <= 2e-5, (name, rel_l2(a, b))


def test_graph_replay_equals_eager():
    model, cams = _setup(seed=5)
    br = batch.BatchRasterizer()
    br.plan(model, cams, gsb.RasterizeOptions(active_sh_degree=3))
    res = br.forward()
    flat, _ = _grad_views(res, seed=1)
    eager = br.backward(flat)
    color = res.color.clone()
    br.capture(flat)
    for _ in range(2):
        br.replay()
        torch.cuda.synchronize()
        assert torch.equal(br.result.color, color)
        assert rel_l2(br.grads.means, eager.means) <= 2e-5
        assert rel_l2(br.grads.sh, eager.sh) <= 2e-5


def test_capacity_overflow_is_reported_not_fatal():
    model, cams = _setup(n=4000, seed=7)
    br = batch.BatchRasterizer()
    br.plan(model, cams, gsb.RasterizeOptions(active_sh_degree=3), instance_capacity=64)
    br.forward()
    info = br.info()
    assert info["overflow"] == 1 and info["instances"] > 64
    assert info["instance_capacity"] == 64


def test_autotune_picks_a_timed_candidate():
    model, cams = _setup(n=8000, seed=9)
    br = batch.BatchRasterizer()
    br.plan(model, cams, gsb.RasterizeOptions(active_sh_degree=3), schedule="auto",
            tune_iterations=1)
    assert len(br.tuning) == 18
    times = [ms for _, ms in br.tuning]
    assert all(np.isfinite(t) and t > 0 for t in times)
    best = min(br.tuning, key=lambda x: x[1])[0]
    assert best == br.schedule
    res = br.forward()
    single, _ = _single(model, cams)
    for v, (c, a, _) in enumerate(single):
        assert float((res.view_color(v) - c).abs().max()) <= 1e-6
