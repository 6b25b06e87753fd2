"""ctypes access to the reference rasterizer and the reference's fused
L1 + SSIM and training-loss kernels, built from their own sources.

TEST INFRASTRUCTURE ONLY (the checker): loads oracle/_ref/libsplat_ref.so,
which oracle/Makefile compiles from the reference's splat_drender sources plus
oracle/ref_harness.cu, oracle/_ref/libssim_ref.so (photara's
fused_ssim.cu plus oracle/ref_ssim_harness.cu), oracle/_ref/libloss_ref.so
(photara's cuda_ops.cu plus oracle/ref_loss_harness.cu) and
oracle/_ref/libprune_ref.so (photara's rasterizer.cu plus
oracle/ref_prune_harness.cu). Only tests/,
__graft_entry__.smoke() and bench.py's reference arm may use it; the product
never does.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libsplat_ref.so"

_lib = None
_synchronous = True


class RefAdam(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "means", "log_scales", "quaternions", "opacity_logits", "means_first", "means_second",
        "scales_first", "scales_second", "rotations_first", "rotations_second", "opacity_first",
        "opacity_second")] + [(n, C.c_float) for n in (
            "means_lr", "scales_lr", "quaternions_lr", "opacities_lr", "beta1", "beta2",
            "correction1", "correction2", "epsilon")] + [
        ("sh_param", C.c_void_p), ("sh_first", C.c_void_p), ("sh_packed", C.c_void_p),
        ("sh_bounds", C.c_void_p)] + [(n, C.c_float) for n in (
            "sh_lr", "sh_rest_lr", "sh_epsilon", "sh_regularization")] + [
        ("sh_stride", C.c_int), ("filter_3d", C.c_void_p)] + [(n, C.c_float) for n in (
            "minimum_log_scale", "maximum_log_scale", "opacity_reg", "scale_reg",
            "shape_erank_reg", "shape_erank_s3_reg", "shape_quat_norm_reg",
            "shape_axis_ratio_reg", "shape_max_axis_ratio")] + [("opacity_gradient", C.c_void_p)]

    def __init__(self, **kw):
        # the reference's StructureAdam defaults (api.h:152-163), then the caller's
        super().__init__(**{**dict(beta1=0.9, beta2=0.999, correction1=1.0, correction2=1.0,
                                   epsilon=1e-15, minimum_log_scale=-1e30,
                                   maximum_log_scale=1e30, shape_max_axis_ratio=100.0), **kw})


def available() -> bool:
    return REF_LIB.exists()


def load():
    global _lib
    if _lib is None:
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} not built (oracle/Makefile ref)")
        lib = C.CDLL(str(REF_LIB))
        vp, f, i = C.c_void_p, C.c_float, C.c_int
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_forward.argtypes = [i, vp, vp, vp, vp, vp, i, i, vp, vp, i, i, f, f, f, f, f, f, i,
                                    f, vp, vp, vp, vp, vp, vp, i, vp, vp]
        lib.ref_forward.restype = i
        lib.ref_forward_ex.argtypes = lib.ref_forward.argtypes + [vp, vp]
        lib.ref_forward_ex.restype = i
        lib.ref_forward_colors.argtypes = [vp, vp, vp, vp]
        lib.ref_forward_colors.restype = i
        lib.ref_backward_ex.argtypes = [vp] * 10 + [C.POINTER(RefAdam), vp]
        lib.ref_backward_ex.restype = i
        lib.ref_draw_list.argtypes = [vp, vp]
        lib.ref_draw_list.restype = i
        lib.ref_forward_state.argtypes = [C.POINTER(vp)] * 4 + [C.POINTER(i)]
        lib.ref_forward_state.restype = i
        lib.ref_backward_geometry.argtypes = [vp] * 13
        lib.ref_backward_geometry.restype = i
        lib.ref_backward_full.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                          C.POINTER(RefAdam)]
        lib.ref_backward_full.restype = i
        lib.ref_set_synchronous.argtypes = [i]
        lib.ref_set_synchronous.restype = None
        _lib = lib
    return _lib


def set_synchronous(on: bool) -> None:
    """True (default): forward/backward wait for the device around each call.
    False: they only enqueue (the reference forward still waits for its draw
    counts); valid when torch's current stream is the legacy default stream,
    on which the reference launches, so the order of torch's work and the
    reference's is the stream's own."""
    global _synchronous
    if not on and torch.cuda.current_stream().cuda_stream != 0:
        raise RuntimeError("asynchronous reference calls need torch on the legacy default stream")
    _synchronous = bool(on)
    load().ref_set_synchronous(1 if on else 0)


def _sync():
    if _synchronous:
        torch.cuda.synchronize()


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference: " + load().ref_last_error().decode())


def forward(model, camera, background=(0.0, 0.0, 0.0), kernel_size=0.0, compensate_2d=True,
            near_plane=0.2, alpha_clip=0.99, sh_degree=3, need_depth=False, filter_3d=None,
            colors=None):
    """Reference forward on the same device tensors. Returns a dict (with
    "median_depth" [H,W] and "normal" [3,H,W] when need_depth). filter_3d:
    [N] Mip-Splatting 3D filter or None; colors: [N,3] precomputed colours in
    place of the SH, or None."""
    lib = load()
    dev = model.means.device
    n = model.means.shape[0]
    H, W = camera.height, camera.width
    color = torch.zeros((3, H, W), device=dev)
    alpha = torch.zeros((H, W), device=dev)
    radii = torch.zeros((n,), device=dev, dtype=torch.int32)
    vis = torch.zeros((n,), device=dev)
    view = (C.c_float * 16)(*[float(v) for v in camera.world_to_camera])
    center = (C.c_float * 3)(*[float(v) for v in camera.position])
    bg = (C.c_float * 3)(*[float(v) for v in background])
    counts = (C.c_int * 2)()
    depth = torch.zeros((H, W), device=dev) if need_depth else None
    normal = torch.zeros((3, H, W), device=dev) if need_depth else None
    _sync()
    _check(lib.ref_forward_ex(n, _p(model.means), _p(model.log_scales), _p(model.quaternions),
                              _p(model.opacity_logits), _p(model.sh), int(sh_degree),
                              int(model.sh.shape[1]), C.cast(view, C.c_void_p),
                              C.cast(center, C.c_void_p), W, H, float(camera.fx),
                              float(camera.fy), float(camera.cx), float(camera.cy),
                              float(near_plane), float(alpha_clip), 1 if compensate_2d else 0,
                              float(kernel_size), C.cast(bg, C.c_void_p), _p(color), _p(alpha),
                              _p(radii), _p(vis), C.cast(counts, C.c_void_p),
                              1 if need_depth else 0, _p(depth) if need_depth else None,
                              _p(normal) if need_depth else None, _p(filter_3d), _p(colors)))
    out = {"color": color, "alpha": alpha, "radii": radii, "visibility": vis,
           "instances": counts[0], "visible": counts[1]}
    if need_depth:
        out["median_depth"], out["normal"] = depth, normal
    return out


def backward_geometry(fwd, grad_color, grad_alpha, grad_depth, grad_normal, n, sh_numel,
                      device, out: dict | None = None):
    """Reference backward of the last reference forward (rendered with
    need_depth=True) including the median-depth and normal output gradients
    (activated-space parameter gradients), accumulated into `out` (zeroed
    buffers allocated here when not given)."""
    lib = load()
    z = lambda *s: torch.zeros(s, device=device)
    if out is None:
        out = {"means": z(n, 3), "sh": torch.zeros(sh_numel, device=device), "opacities": z(n),
               "scales": z(n, 3), "rotations": z(n, 4)}
    if "median_depth" not in fwd or "normal" not in fwd:
        raise ValueError("the geometry backward needs a forward rendered with need_depth=True")
    _sync()
    _check(lib.ref_backward_geometry(_p(fwd["alpha"]), _p(fwd["radii"]),
                                     _p(fwd["median_depth"]), _p(fwd["normal"]), _p(grad_color),
                                     _p(grad_alpha), _p(grad_depth), _p(grad_normal),
                                     _p(out["means"]), _p(out["sh"]), _p(out["opacities"]),
                                     _p(out["scales"]), _p(out["rotations"])))
    return out


def forward_colors(fwd, colors):
    """Rasterizer::forward_colors (pipeline.cu:617-649) over the last reference
    forward (rendered from colours): new colour and alpha images."""
    lib = load()
    dev = colors.device
    H, W = fwd["alpha"].shape
    out = {"color": torch.zeros((3, H, W), device=dev), "alpha": torch.zeros((H, W), device=dev),
           "visibility": torch.zeros_like(fwd["visibility"])}
    _sync()
    _check(lib.ref_forward_colors(_p(colors), _p(out["color"]), _p(out["alpha"]),
                                  _p(out["visibility"])))
    return {**fwd, **out}


def draw_list(instances, width, height, device):
    lib = load()
    tiles = ((width + 15) // 16) * ((height + 15) // 16)
    vals = torch.zeros((max(instances, 1),), dtype=torch.int32, device=device)
    ranges = torch.zeros((tiles, 2), dtype=torch.int32, device=device)
    _check(lib.ref_draw_list(_p(vals), _p(ranges)))
    torch.cuda.synchronize()
    return vals[:instances], ranges


def backward(fwd, grad_color, grad_alpha, n, sh_numel, device, adam: RefAdam | None = None,
             out: dict | None = None, colors: bool = False):
    """Reference backward of the last reference forward (activated-space grads),
    accumulated into `out` (zeroed buffers allocated here when not given).
    colors: the forward was rendered from precomputed colours; their gradient
    comes back as out["colors"] [N,3] (and no SH gradient)."""
    lib = load()
    z = lambda *s: torch.zeros(s, device=device)
    if out is None:
        out = {"means": z(n, 3), "sh": None if colors else torch.zeros(sh_numel, device=device),
               "opacities": z(n), "scales": z(n, 3), "rotations": z(n, 4),
               "refine_weight": z(n), "colors": z(n, 3) if colors else None}
    _sync()
    _check(lib.ref_backward_ex(_p(fwd["alpha"]), _p(fwd["radii"]), _p(grad_color),
                               _p(grad_alpha), _p(out["means"]), _p(out.get("sh")),
                               _p(out["opacities"]), _p(out["scales"]), _p(out["rotations"]),
                               _p(out["refine_weight"]), C.byref(adam) if adam else None,
                               _p(out.get("colors"))))
    return out


# --- the reference's fused L1 + SSIM kernels (oracle/_ref/libssim_ref.so) ---

SSIM_LIB = HERE / "_ref" / "libssim_ref.so"
_ssim = None


def ssim_available() -> bool:
    return SSIM_LIB.exists()


def _ssim_lib():
    global _ssim
    if _ssim is None:
        if not SSIM_LIB.exists():
            raise RuntimeError(f"{SSIM_LIB} not built (oracle/Makefile ref)")
        lib = C.CDLL(str(SSIM_LIB))
        vp, f, i = C.c_void_p, C.c_float, C.c_int
        lib.ref_fused_l1_ssim.argtypes = [vp, vp, vp, f, f, vp, vp, i, i, vp]
        lib.ref_fused_l1_ssim.restype = i
        lib.ref_ssim_metric.argtypes = [vp, vp, vp, i, i, vp, vp]
        lib.ref_ssim_metric.restype = i
        _ssim = lib
    return _ssim


def fused_l1_ssim(prediction, target, mask=None, ssim_weight=0.2, photometric_weight=1.0,
                  grad=None, loss=None):
    """cuda_backend::fused_l1_ssim_loss on device tensors ([3,H,W], mask [H,W]):
    adds the gradient into `grad` and the loss into `loss` ([1]), both
    allocated zeroed when not given. Returns (loss, grad)."""
    H, W = int(prediction.shape[1]), int(prediction.shape[2])
    grad = torch.zeros_like(prediction) if grad is None else grad
    loss = torch.zeros((1,), device=prediction.device) if loss is None else loss
    stream = torch.cuda.current_stream(prediction.device).cuda_stream
    rc = _ssim_lib().ref_fused_l1_ssim(_p(prediction), _p(target), _p(mask), float(ssim_weight),
                                       float(photometric_weight), _p(grad), _p(loss), W, H,
                                       C.c_void_p(stream))
    if rc != 0:
        raise RuntimeError(f"reference fused SSIM failed ({rc})")
    return loss, grad


def ssim_metric(prediction, target, mask=None) -> float:
    """cuda_backend::fused_ssim_metric on device tensors."""
    H, W = int(prediction.shape[1]), int(prediction.shape[2])
    out = torch.zeros((1,), device=prediction.device)
    stream = torch.cuda.current_stream(prediction.device).cuda_stream
    rc = _ssim_lib().ref_ssim_metric(_p(prediction), _p(target), _p(mask), W, H, _p(out),
                                     C.c_void_p(stream))
    if rc != 0:
        raise RuntimeError(f"reference SSIM metric failed ({rc})")
    return float(out)


# --- the reference's training-loss kernels (oracle/_ref/libloss_ref.so) ---

LOSS_LIB = HERE / "_ref" / "libloss_ref.so"
_loss = None


def loss_available() -> bool:
    return LOSS_LIB.exists() and SSIM_LIB.exists()


def _loss_lib():
    global _loss
    if _loss is None:
        if not LOSS_LIB.exists():
            raise RuntimeError(f"{LOSS_LIB} not built (oracle/Makefile ref)")
        lib = C.CDLL(str(LOSS_LIB))
        vp, f, i = C.c_void_p, C.c_float, C.c_int
        lib.ref_loss_kernel.argtypes = [vp] * 13 + [C.c_size_t, f, f, f, i, i, f, f, i, vp]
        lib.ref_loss_kernel.restype = i
        lib.ref_depth_normal.argtypes = [vp] * 5 + [C.c_uint, C.c_uint, f, f, f, f, f, vp]
        lib.ref_depth_normal.restype = i
        lib.ref_split_gaussians.argtypes = [vp] * 10 + [C.c_size_t, i, f, f, f, vp]
        lib.ref_split_gaussians.restype = i
        lib.ref_adc_decay.argtypes = [vp, vp, C.c_size_t, f, f, vp]
        lib.ref_adc_decay.restype = i
        lib.ref_accumulate_densification.argtypes = [vp] * 7 + [C.c_size_t, f, i, i, f, f] + \
            [vp] * 4 + [i] + [vp] * 3 + [vp]
        lib.ref_accumulate_densification.restype = i
        _loss = lib
    return _loss


def training_loss(color, target_color, *, alpha=None, median_depth=None, normal=None,
                  target_depth=None, target_normal=None, mask=None, intrinsics=None,
                  photometric_weight=1.0, ssim_weight=0.2, depth_weight=0.0, normal_weight=0.0,
                  depth_normal_weight=0.0, match_alpha_weight=0.25, geometry_epsilon=1e-3,
                  alpha_mode="masked", ai_prior=False, need_geometry_gradients=False):
    """cuda_backend::compute_training_loss (cuda_ops.cu:2731-2822) on device
    tensors, through the reference's own kernels: loss_kernel, the fused
    SSIM kernels when the image is > 10 pixels across, then the depth-normal
    consistency kernel. Returns a dict like oracle.loss_ref.training_loss."""
    H, W = int(color.shape[1]), int(color.shape[2])
    dev = color.device
    out = {"color": torch.empty_like(color), "alpha": torch.empty((H, W), device=dev),
           "depth": torch.empty((H, W), device=dev) if need_geometry_gradients else None,
           "normal": torch.empty((3, H, W), device=dev) if need_geometry_gradients else None,
           "terms": torch.zeros((4,), device=dev)}
    modes = {"validity": -1, "masked": 0, "transparent": 1}
    fused = W > 10 and H > 10
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    lib = _loss_lib()
    rc = lib.ref_loss_kernel(_p(color), _p(alpha), _p(median_depth), _p(normal),
                             _p(target_color), _p(target_depth), _p(target_normal), _p(mask),
                             _p(out["color"]), _p(out["alpha"]), _p(out["depth"]),
                             _p(out["normal"]), _p(out["terms"]), H * W,
                             0.0 if fused else float(photometric_weight), float(depth_weight),
                             float(normal_weight), 1 if mask is not None else 0,
                             modes[alpha_mode], float(match_alpha_weight),
                             float(geometry_epsilon), 1 if ai_prior else 0, stream)
    if rc != 0:
        raise RuntimeError(f"reference loss kernel failed ({rc})")
    if fused:
        fused_l1_ssim(color, target_color, mask, min(max(ssim_weight, 0.0), 1.0),
                      photometric_weight, grad=out["color"], loss=out["terms"])
    if need_geometry_gradients and depth_normal_weight > 0:
        fx, fy, cx, cy = intrinsics
        rc = lib.ref_depth_normal(_p(median_depth), _p(normal), _p(out["depth"]),
                                  _p(out["normal"]), _p(out["terms"]), W, H, float(fx), float(fy),
                                  float(cx), float(cy), float(depth_normal_weight), stream)
        if rc != 0:
            raise RuntimeError(f"reference depth-normal kernel failed ({rc})")
    return out


def l1_loss(color, target_color, grad_color, grad_alpha, terms, weight=1.0):
    """The reference's L1 photometric term alone: loss_kernel
    (cuda_ops.cu:846-891) with photo_weight = weight and every other term off,
    no mask. Writes grad_color = weight/(3P) sign(color - target), zeroes
    grad_alpha, and, when terms is given, adds weight/(3P) sum|color - target|
    into terms[0] (one atomic per pixel, as the reference does; terms = None
    skips the scalar)."""
    H, W = int(color.shape[1]), int(color.shape[2])
    stream = C.c_void_p(torch.cuda.current_stream(color.device).cuda_stream)
    rc = _loss_lib().ref_loss_kernel(_p(color), None, None, None, _p(target_color), None, None,
                                     None, _p(grad_color), _p(grad_alpha), None, None, _p(terms),
                                     H * W, float(weight), 0.0, 0.0, 0, 0, 0.25, 1e-3, 0, stream)
    if rc != 0:
        raise RuntimeError(f"reference loss kernel failed ({rc})")


SPLIT_MODES = {"adc_covariance": 0, "dense_tangent": 1, "igs_random": 2, "long_axis": 3}


def split_gaussians(parent, child, parent_indices, mode, random_samples=None, screen_sizes=None,
                    minimum_opacity=1e-6, split_at_screen_size=0.0, split_opacity_k=0.5):
    """cuda_backend::split_gaussians (cuda_ops.cu:3105) on dicts of device
    tensors (means, log_scales, opacity_logits, quaternions), in place."""
    stream = C.c_void_p(torch.cuda.current_stream(parent["means"].device).cuda_stream)
    rc = _loss_lib().ref_split_gaussians(
        _p(parent["means"]), _p(parent["log_scales"]), _p(parent["opacity_logits"]),
        _p(parent["quaternions"]), _p(child["means"]), _p(child["log_scales"]),
        _p(child["opacity_logits"]), _p(parent_indices), _p(random_samples), _p(screen_sizes),
        parent_indices.numel(), SPLIT_MODES[mode], float(minimum_opacity),
        float(split_at_screen_size), float(split_opacity_k), stream)
    if rc != 0:
        raise RuntimeError(f"reference split failed ({rc})")


def adc_decay(log_scales, opacity_logits, opacity_decay, scale_decay):
    """cuda_backend::apply_adc_decay (cuda_ops.cu:3388), in place."""
    stream = C.c_void_p(torch.cuda.current_stream(log_scales.device).cuda_stream)
    rc = _loss_lib().ref_adc_decay(_p(log_scales), _p(opacity_logits), opacity_logits.numel(),
                                   float(opacity_decay), float(scale_decay), stream)
    if rc != 0:
        raise RuntimeError(f"reference ADC decay failed ({rc})")


def accumulate_densification(stats, refine_weight, visibility, radii, inverse_resolution,
                             use_maximum=True, require_visibility=True, step_score_power=1.0,
                             oversize_screen_threshold=0.0, geometry_gradient=None,
                             view_index=-1, image_error=None, normalized_size=None):
    """accumulate_densification_kernel (cuda_ops.cu:1548-1606) on the dict of
    device statistics `stats` (gradient, count, max_screen_radius, priority,
    max_geometry_gradient, first_view (int32), view_support, image_error), in
    place."""
    stream = C.c_void_p(torch.cuda.current_stream(radii.device).cuda_stream)
    rc = _loss_lib().ref_accumulate_densification(
        _p(refine_weight), _p(visibility), _p(radii), _p(stats["gradient"]), _p(stats["count"]),
        _p(stats["max_screen_radius"]), _p(stats["priority"]), radii.numel(),
        float(inverse_resolution), 1 if use_maximum else 0, 1 if require_visibility else 0,
        float(step_score_power), float(oversize_screen_threshold), _p(geometry_gradient),
        _p(stats["max_geometry_gradient"]), _p(stats["first_view"]), _p(stats["view_support"]),
        int(view_index), _p(image_error), _p(stats["image_error"]), _p(normalized_size), stream)
    if rc != 0:
        raise RuntimeError(f"reference densification accumulate failed ({rc})")


# --- the reference's Speedy-Splat score kernel (oracle/_ref/libprune_ref.so) ---

PRUNE_LIB = HERE / "_ref" / "libprune_ref.so"
_prune = None


def prune_available() -> bool:
    return PRUNE_LIB.exists() and REF_LIB.exists()


def pruning_scores(model, camera, background=(0.0, 0.0, 0.0), alpha_clip=0.99,
                   gaussian_pop=False, sh_degree=3):
    """CudaRasterizer::pruning_scores (rasterizer.cu:450-490): a reference
    forward, then the reference's sensitivity_scores kernel over its
    workspace. Returns (scores [N], forward dict)."""
    global _prune
    lib = load()
    if _prune is None:
        if not PRUNE_LIB.exists():
            raise RuntimeError(f"{PRUNE_LIB} not built (oracle/Makefile ref)")
        pl = C.CDLL(str(PRUNE_LIB))
        vp, f, i = C.c_void_p, C.c_float, C.c_int
        pl.ref_sensitivity_scores.argtypes = [i, i, vp, C.c_size_t, vp, vp, vp, vp, vp, f, i, vp]
        pl.ref_sensitivity_scores.restype = i
        _prune = pl
    fwd = forward(model, camera, background=background, alpha_clip=alpha_clip,
                  sh_degree=sh_degree)
    n = model.means.shape[0]
    scores = torch.zeros((n,), device=model.means.device)
    if fwd["instances"] == 0:
        return scores, fwd
    ptrs = [C.c_void_p() for _ in range(4)]
    inst = C.c_int()
    _check(lib.ref_forward_state(*[C.byref(q) for q in ptrs], C.byref(inst)))
    stream = C.c_void_p(torch.cuda.current_stream(model.means.device).cuda_stream)
    rc = _prune.ref_sensitivity_scores(camera.width, camera.height, ptrs[0], n, ptrs[1], ptrs[3],
                                       ptrs[2], _p(fwd["color"]), _p(scores), float(alpha_clip),
                                       1 if gaussian_pop else 0, stream)
    if rc != 0:
        raise RuntimeError(f"reference pruning scores failed ({rc})")
    return scores, fwd
