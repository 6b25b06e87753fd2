"""ctypes binding of libgsplat_b200.so (include/gsplat_b200.h).

The structs below mirror the header field for field. Loading fails loudly when
the library is missing: there is no CPU or Python fallback for the rasterizer.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libgsplat_b200.so"

GS_OK, GS_ERR_INVALID, GS_ERR_CUDA, GS_ERR_STATE, GS_ERR_CAPACITY, GS_ERR_TIMEOUT = range(6)

fp = C.POINTER(C.c_float)
vp = C.c_void_p


class Gaussians(C.Structure):
    _fields_ = [("count", C.c_int), ("means", vp), ("log_scales", vp), ("quaternions", vp),
                ("opacity_logits", vp), ("filter_3d", vp), ("sh", vp), ("colors", vp),
                ("sh_degree", C.c_int), ("sh_bases", C.c_int)]


class Camera(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("fx", C.c_float), ("fy", C.c_float),
                ("cx", C.c_float), ("cy", C.c_float), ("near_plane", C.c_float),
                ("alpha_clip", C.c_float), ("compensate_2d", C.c_int),
                ("world_to_camera", C.c_float * 16), ("center", C.c_float * 3)]


class Settings(C.Structure):
    _fields_ = [("background", C.c_float * 3), ("scale_modifier", C.c_float),
                ("kernel_size", C.c_float), ("record_backward_state", C.c_int),
                ("need_depth", C.c_int)]


class Outputs(C.Structure):
    _fields_ = [("color", vp), ("alpha", vp), ("visibility", vp), ("radii", vp),
                ("median_depth", vp), ("normal", vp)]


class ForwardInfo(C.Structure):
    _fields_ = [("instance_count", C.c_int), ("visible_count", C.c_int), ("depth_bits", C.c_int),
                ("tile_bits", C.c_int), ("tiles", C.c_int)]


class LossGrads(C.Structure):
    _fields_ = [("color", vp), ("alpha", vp), ("densify_map", vp), ("median_depth", vp),
                ("normal", vp)]


class LossImages(C.Structure):
    _fields_ = [(n, vp) for n in ("color", "alpha", "median_depth", "normal", "target_color",
                                  "target_depth", "target_normal", "mask")] + [
        ("width", C.c_int), ("height", C.c_int), ("fx", C.c_float), ("fy", C.c_float),
        ("cx", C.c_float), ("cy", C.c_float)]


class LossOptions(C.Structure):
    _fields_ = [(n, C.c_float) for n in (
        "photometric_weight", "ssim_weight", "depth_weight", "normal_weight",
        "depth_normal_weight", "match_alpha_weight", "geometry_epsilon")] + [
        ("mask_enabled", C.c_int), ("alpha_mode", C.c_int), ("ai_prior", C.c_int)]


class LossOutputs(C.Structure):
    _fields_ = [(n, vp) for n in ("grad_color", "grad_alpha", "grad_depth", "grad_normal",
                                  "terms")]


class DensifyAccum(C.Structure):
    _fields_ = [(n, vp) for n in (
        "refine_weight", "visibility", "radii", "gradient", "count", "max_screen_radius",
        "priority", "geometry_gradient", "max_geometry_gradient", "first_view", "view_support",
        "image_error", "accumulated_error", "normalized_size")] + [
        ("count_rows", C.c_int), ("inverse_resolution", C.c_float), ("use_maximum", C.c_int),
        ("require_visibility", C.c_int), ("step_score_power", C.c_float),
        ("oversize_screen_threshold", C.c_float), ("view_index", C.c_int)]


class SplitArgs(C.Structure):
    _fields_ = [(n, vp) for n in (
        "parent_means", "parent_log_scales", "parent_opacity_logits", "parent_quaternions",
        "child_means", "child_log_scales", "child_opacity_logits", "parents", "random_samples",
        "screen_sizes")] + [("count", C.c_int), ("mode", C.c_int), ("minimum_opacity", C.c_float),
                            ("split_at_screen_size", C.c_float), ("split_opacity_k", C.c_float)]


class ModelGrads(C.Structure):
    _fields_ = [("means", vp), ("scales", vp), ("rotations", vp), ("opacities", vp), ("sh", vp),
                ("colors", vp), ("refine_weight", vp), ("densify_weight", vp),
                ("densify_weight_den", vp), ("activated", C.c_int)]


class StructureAdam(C.Structure):
    _fields_ = [(n, vp) for n in (
        "means", "log_scales", "quaternions", "opacity_logits", "means_first", "means_second",
        "scales_first", "scales_second", "rotations_first", "rotations_second", "opacity_first",
        "opacity_second", "filter_3d")] + [(n, C.c_float) for n in (
            "means_lr", "scales_lr", "quaternions_lr", "opacities_lr", "beta1", "beta2",
            "correction1", "correction2", "epsilon", "minimum_log_scale", "maximum_log_scale",
            "opacity_reg", "scale_reg", "shape_erank_reg", "shape_erank_s3_reg",
            "shape_quat_norm_reg", "shape_axis_ratio_reg", "shape_max_axis_ratio")] + [
        ("opacity_gradient", vp)]


class ShAdam(C.Structure):
    _fields_ = [("parameter", vp)] + [(n, C.c_float) for n in (
        "lr", "rest_lr", "beta1", "beta2", "correction1", "correction2", "epsilon",
        "regularization_factor")] + [("first", vp), ("packed", vp), ("bounds", vp),
                                     ("stride", C.c_int)]


class DensifyStats(C.Structure):
    _fields_ = [(n, vp) for n in ("grad_acc", "count", "max_screen", "err_num", "err_den",
                                        "depth_acc", "age")]


class AdcParams(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("grad_threshold", "percent_dense", "extent",
                                          "prune_opacity", "prune_world_scale", "prune_screen")] + [
        ("densify", C.c_int)]


class BatchSchedule(C.Structure):
    _fields_ = [("tile_w", C.c_int), ("tile_h", C.c_int), ("pixels_per_thread", C.c_int),
                ("schedule", C.c_int), ("ctas_per_sm", C.c_int)]


class BatchInfo(C.Structure):
    _fields_ = [("pairs", C.c_size_t), ("instance_capacity", C.c_size_t),
                ("total_pixels", C.c_size_t), ("total_tiles", C.c_int), ("views", C.c_int),
                ("instances", C.c_longlong), ("visible", C.c_int), ("overflow", C.c_int),
                ("device_error", C.c_int)]


# Every symbol include/gsplat_b200.h declares, with its ctypes signature.
SIGNATURES = {
    "gs_abi_version": ([], C.c_int),
    "gs_create": ([C.POINTER(vp), C.c_int, vp], C.c_int),
    "gs_destroy": ([vp], None),
    "gs_set_stream": ([vp, vp], C.c_int),
    "gs_last_error": ([vp], C.c_char_p),
    "gs_workspace_bytes": ([vp], C.c_size_t),
    "gs_forward": ([vp, C.POINTER(Gaussians), C.POINTER(Camera), C.POINTER(Settings),
                    C.POINTER(Outputs), C.POINTER(ForwardInfo)], C.c_int),
    "gs_backward": ([vp, vp, vp, C.POINTER(LossGrads), C.POINTER(ModelGrads),
                     C.POINTER(StructureAdam), C.POINTER(ShAdam)], C.c_int),
    "gs_set_schedule": ([vp, C.c_int], C.c_int),
    "gs_debug_draw_list": ([vp, vp, vp, vp], C.c_int),
    "gs_enable_stage_timing": ([vp, C.c_int], C.c_int),
    "gs_stage_times": ([vp, fp, C.c_int], C.c_int),
    "gs_exclusive_scan_u32": ([vp, vp, vp, C.c_int, vp], C.c_int),
    "gs_exclusive_scan_u32_noalloc": ([vp, vp, C.c_int, vp, vp], C.c_int),
    "gs_exclusive_scan_u32_noalloc_status": ([vp, vp], C.c_int),
    "gs_device_status": ([vp], C.c_int),
    "gs_debug_lookback_probe": ([vp, C.c_int, C.c_uint], C.c_int),
    "gs_debug_composite_pairs": ([vp, vp, vp, C.POINTER(C.c_ulonglong)], C.c_int),
    "gs_accumulate_densification": ([vp, C.POINTER(DensifyAccum)], C.c_int),
    "gs_sort_pairs_u64": ([vp, vp, vp, vp, vp, C.c_size_t, C.c_int, C.c_int], C.c_int),
    "gs_densify_accumulate": ([vp, C.c_int, vp, vp, vp, vp, C.c_float, vp, fp,
                               C.POINTER(DensifyStats)], C.c_int),
    "gs_densify_features": ([vp, C.c_int, vp, vp, vp, vp, C.c_int, C.POINTER(DensifyStats), fp,
                             C.c_float, vp, vp], C.c_int),
    "gs_adc_decide": ([vp, C.c_int, vp, vp, C.POINTER(DensifyStats), C.POINTER(AdcParams), vp],
                      C.c_int),
    "gs_proposal_policy": ([vp, C.c_int, vp, vp, C.POINTER(DensifyStats), C.c_float, vp],
                           C.c_int),
    "gs_split_gaussians": ([vp, C.c_int, vp, C.c_int, vp, vp, vp, vp], C.c_int),
    "gs_mlp_param_count": ([], C.c_int),
    "gs_mlp_forward": ([vp, C.c_int, vp, vp, vp], C.c_int),
    "gs_mlp_train_step": ([vp, C.c_int, vp, vp, vp, vp, C.c_float, vp, vp], C.c_int),
    "gs_mlp_adam": ([vp, vp, vp, vp, vp, vp] + [C.c_float] * 6, C.c_int),
    "gs_l1_loss": ([vp, vp, vp, C.c_int, C.c_float, vp, vp], C.c_int),
    "gs_fused_l1_ssim": ([vp, vp, vp, vp, C.c_int, C.c_int, C.c_float, C.c_float, vp, vp],
                         C.c_int),
    "gs_ssim_metric": ([vp, vp, vp, vp, C.c_int, C.c_int, vp], C.c_int),
    "gs_training_loss": ([vp, C.POINTER(LossImages), C.POINTER(LossOptions),
                          C.POINTER(LossOutputs)], C.c_int),
    "gs_split_gaussians_mode": ([vp, C.POINTER(SplitArgs)], C.c_int),
    "gs_pruning_scores": ([vp, vp, C.c_int, vp], C.c_int),
    "gs_forward_colors": ([vp, vp, C.POINTER(Outputs)], C.c_int),
    "gs_adc_decay": ([vp, C.c_size_t, vp, vp, C.c_float, C.c_float], C.c_int),
    "gs_select_rows": ([vp, C.c_int, vp, vp, vp], C.c_int),
    "gs_gather_rows": ([vp, C.c_int, vp, C.c_int, C.POINTER(vp), C.POINTER(vp),
                        C.POINTER(C.c_size_t)], C.c_int),
    "gs_adam": ([vp, vp, vp, vp, vp, C.c_size_t] + [C.c_float] * 8, C.c_int),
    "gs_batch_create": ([C.POINTER(vp), C.c_int, vp], C.c_int),
    "gs_batch_destroy": ([vp], None),
    "gs_batch_last_error": ([vp], C.c_char_p),
    "gs_batch_set_stream": ([vp, vp], C.c_int),
    "gs_batch_plan": ([vp, C.POINTER(Gaussians), C.POINTER(Camera), C.c_int, C.POINTER(Settings),
                       C.POINTER(BatchSchedule), C.c_size_t], C.c_int),
    "gs_batch_get_info": ([vp, C.POINTER(BatchInfo)], C.c_int),
    "gs_batch_forward": ([vp, vp, vp, vp], C.c_int),
    "gs_batch_backward": ([vp, vp, vp, C.POINTER(ModelGrads)], C.c_int),
    "gs_batch_capture": ([vp, vp, vp, vp, vp, vp, C.POINTER(ModelGrads)], C.c_int),
    "gs_batch_replay": ([vp], C.c_int),
    "gs_batch_autotune": ([vp, C.POINTER(Gaussians), C.POINTER(Camera), C.c_int,
                           C.POINTER(Settings), C.c_int, C.POINTER(BatchSchedule), fp,
                           C.POINTER(BatchSchedule), fp, C.POINTER(C.c_int)], C.c_int),
}

_lib = None


def load() -> C.CDLL:
    """Loads the library once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | C.RTLD_GLOBAL)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


class GsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class InvalidArgument(GsError, ValueError):
    pass


class StateError(GsError):
    pass


def check(status: int, ctx, batch: bool = False) -> None:
    """Raises the exception matching a gs_status (message from the context,
    or from the batch handle when `batch`)."""
    if status == GS_OK:
        return
    lib = load()
    getter = lib.gs_batch_last_error if batch else lib.gs_last_error
    msg = getter(ctx).decode() if ctx else "gsplat_b200 error"
    if status == GS_ERR_INVALID:
        raise InvalidArgument(status, msg)
    if status == GS_ERR_STATE:
        raise StateError(status, msg)
    raise GsError(status, msg)
