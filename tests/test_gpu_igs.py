"""ADC-IGS on the GPU: the densification statistics kernel against the
reference's own accumulate_densification_kernel (photara/src/splat/cuda_ops.cu
:1548-1606, built into oracle/_ref/libloss_ref.so), and one IGS refinement
applied to a model with its Adam state (igs.apply_igs).

The statistics are integer counts and float running maxima / sums of the same
float32 values in the same order per row, so they must be identical."""
import importlib

import numpy as np
import pytest
import torch

from helpers import camera_of, device_model, gsb

ref = pytest.importorskip("oracle.reference")
igs = importlib.import_module("photara-studio_b200.igs")
densify = importlib.import_module("photara-studio_b200.densify")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]


def _stats_dict(n):
    z = lambda: torch.zeros(n, device="cuda")
    return {"gradient": z(), "count": z(), "max_screen_radius": z(), "priority": z(),
            "max_geometry_gradient": z(), "view_support": z(), "image_error": z(),
            "first_view": torch.zeros(n, dtype=torch.int32, device="cuda")}


@pytest.mark.parametrize("use_max,threshold,power,with_error", [
    (True, 0.25, 1.0, False), (False, 0.0, 1.0, True), (True, 0.0, 0.5, True),
    (False, 0.1, 2.0, False)])
def test_accumulate_matches_reference_kernel(use_max, threshold, power, with_error):
    if not ref.loss_available():
        pytest.skip("reference loss kernels not built (oracle/_ref)")
    n = 50_000
    g = torch.Generator(device="cuda").manual_seed(7)
    ours, theirs = _stats_dict(n), _stats_dict(n)
    lib = gsb.load_library()
    for view in range(5):
        rw = torch.rand(n, device="cuda", generator=g) * 0.01
        rw[::97] = float("nan")
        rw[::89] = -1.0
        vis = (torch.rand(n, device="cuda", generator=g) > 0.3).float()
        radii = (torch.rand(n, device="cuda", generator=g) * 60).int()
        radii[::7] = 0
        err = torch.rand(n, device="cuda", generator=g) if with_error else None
        view_index = view % 3 if view < 4 else -1
        ref.accumulate_densification(theirs, rw, vis, radii, 1.0 / 720, use_maximum=use_max,
                                     require_visibility=True, step_score_power=power,
                                     oversize_screen_threshold=threshold, geometry_gradient=rw,
                                     view_index=view_index, image_error=err)
        a = gsb._lib.DensifyAccum()
        a.refine_weight, a.visibility, a.radii = rw.data_ptr(), vis.data_ptr(), radii.data_ptr()
        for k in ("gradient", "count", "max_screen_radius", "priority", "max_geometry_gradient",
                  "view_support"):
            setattr(a, k, ours[k].data_ptr())
        a.geometry_gradient = rw.data_ptr()
        a.first_view = ours["first_view"].data_ptr()
        a.image_error = err.data_ptr() if err is not None else None
        a.accumulated_error = ours["image_error"].data_ptr()
        a.count_rows = n
        a.inverse_resolution = 1.0 / 720
        a.use_maximum, a.require_visibility = int(use_max), 1
        a.step_score_power, a.oversize_screen_threshold = power, threshold
        a.view_index = view_index
        ctx = gsb.rasterizer._pool(0).take()
        ctx.bind_stream()
        try:
            assert lib.gs_accumulate_densification(ctx.ptr, a) == 0
        finally:
            ctx.release()
    torch.cuda.synchronize()
    for k in ours:
        assert torch.equal(ours[k], theirs[k]), k


def test_igs_refinement_applies_plan_to_model_and_adam_state():
    scene = gsb.make_scene("g16k_256", seed=3)
    model = device_model(scene)
    model.opacity_logits[::50] = -8.0   # below the 1/255 floor: recycled
    cam = camera_of(scene)
    n = model.size()
    opts = igs.IgsOptions(dense_recycle_fraction=0.05)
    stats = igs.IgsStats(n, "cuda")
    adam = densify.AdamState.zeros(model)
    for k in adam.structure:
        adam.structure[k].fill_(0.5)
    rast = gsb.Rasterizer()
    r = rast.forward(model, cam, gsb.RasterizeOptions(active_sh_degree=3))
    grads = rast.backward(model, r, torch.full_like(r.color, 1e-3), None)
    stats.accumulate(r, grads.refine_weight, cam, model.means, 0, opts)
    g = torch.Generator(device="cuda").manual_seed(0)
    plan = igs.igs_plan(model, stats, 1000, opts, extent=6.0, center=(0, 0, 0), gen=g)
    assert plan.pruned > 0 and plan.parents.numel() > 0
    before = {f: getattr(model, f).clone() for f in ("means", "log_scales", "opacity_logits")}
    screen = stats.t["max_screen_radius"].clone()
    m2, a2, info = igs.apply_igs(model, adam, stats, plan, screen, 1000, opts, g)
    torch.cuda.synchronize()
    kept = int(plan.keep.sum())
    npar = plan.parents.numel()
    assert m2.size() == kept + npar == info["count"]
    keep_idx = torch.nonzero(plan.keep).flatten()
    is_parent = torch.zeros(kept, dtype=torch.bool, device="cuda")
    is_parent[plan.parents] = True
    # survivors that are not parents keep their means and moments
    plain = ~is_parent
    assert torch.equal(m2.means[:kept][plain], before["means"][keep_idx][plain])
    assert torch.all(a2.structure["means_first"][:kept][plain] == 0.5)
    # parents and children restart their moments; children sit beside parents
    assert torch.all(a2.structure["means_first"][:kept][is_parent] == 0)
    assert torch.all(a2.structure["means_first"][kept:] == 0)
    assert torch.all(a2.sh["packed"][kept:] == 0)
    par_old = keep_idx[plan.parents]
    mid = 0.5 * (m2.means[keep_idx.numel():] + m2.means[:kept][is_parent])
    assert torch.allclose(mid, before["means"][par_old], atol=1e-5)
    assert stats.t["count"].numel() == m2.size()
