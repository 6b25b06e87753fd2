"""Host-side mirror of photara's splat rasterizer interface on torch tensors.

Same names, argument meaning and error behaviour as
  photara::splat::Rasterizer::forward / backward   photara/include/splat/rasterizer.hpp:128,156
  RasterizeOptions / RasterizationPolicy          photara/include/splat/rasterizer.hpp:9-55,
                                                  photara/include/splat/options.hpp:32-37
  GaussianModel / Camera / ModelGradients         photara/include/splat/types.hpp:17-80
  SHAdamUpdate / StructureAdamUpdate              photara/include/splat/rasterizer.hpp:73-104
and the bridge's validation (photara/src/splat/rasterizer.cu:306-329, :495-560).
Every call goes through the C ABI of libgsplat_b200.so; torch only provides
device memory and the current CUDA stream.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
from dataclasses import dataclass, field, replace
from typing import Optional, Sequence

import torch

from . import _lib as L

__all__ = [
    "Camera", "GaussianModel", "RasterizationPolicy", "RasterizeOptions", "RenderResult",
    "ModelGradients", "SHAdamUpdate", "StructureAdamUpdate", "Rasterizer", "look_at_camera",
]


# ------------------------------------------------------------------ types --
@dataclass
class Camera:
    """Pinhole camera; world_to_camera is 16 floats column-major (types.hpp:17-33)."""
    world_to_camera: Sequence[float]
    position: Sequence[float]
    fx: float
    fy: float
    cx: float
    cy: float
    width: int
    height: int


@dataclass
class GaussianModel:
    means: torch.Tensor           # [N,3]
    log_scales: torch.Tensor      # [N,3]
    quaternions: torch.Tensor     # [N,4] scalar-first
    opacity_logits: torch.Tensor  # [N,1] or [N]
    sh: torch.Tensor              # [N,K,3]
    sh_degree: int = 3
    filter_3d: Optional[torch.Tensor] = None  # [N,1]

    def size(self) -> int:
        return int(self.means.shape[0]) if self.means is not None and self.means.dim() > 0 else 0


@dataclass
class RasterizationPolicy:
    alpha_clip: float = 0.99
    near_plane: float = 0.2
    pixel_center_offset: float = 0.0
    compensate_2d: bool = True


@dataclass
class RasterizeOptions:
    rasterization: RasterizationPolicy = field(default_factory=RasterizationPolicy)
    active_sh_degree: int = 0
    background: Sequence[float] = (0.0, 0.0, 0.0)
    kernel_size: float = 0.0
    scale_modifier: float = 1.0
    # photara's default is True; here the median-depth and normal channels are
    # rendered only on request (they re-walk every tile's list five times).
    require_depth: bool = False
    record_backward_state: bool = True
    colors_precomp: Optional[torch.Tensor] = None


@dataclass
class SHAdamUpdate:
    first: torch.Tensor            # [N,K,3] float16
    packed: torch.Tensor           # [N,K,3] uint8
    bounds: torch.Tensor           # [N,4] float32
    lr: float = 0.0
    rest_lr: float = 0.0
    beta1: float = 0.9
    beta2: float = 0.999
    correction1: float = 1.0
    correction2: float = 1.0
    epsilon: float = 1e-8
    regularization_weight: float = 0.0


@dataclass
class StructureAdamUpdate:
    means_first: torch.Tensor
    means_second: torch.Tensor
    scales_first: torch.Tensor
    scales_second: torch.Tensor
    rotations_first: torch.Tensor
    rotations_second: torch.Tensor
    opacity_first: torch.Tensor
    opacity_second: torch.Tensor
    means_lr: float = 0.0
    scales_lr: float = 0.0
    quaternions_lr: float = 0.0
    opacities_lr: float = 0.0
    beta1: float = 0.9
    beta2: float = 0.999
    correction1: float = 1.0
    correction2: float = 1.0
    epsilon: float = 1e-15
    minimum_log_scale: float = -math.inf
    maximum_log_scale: float = math.inf
    opacity_reg: float = 0.0
    scale_reg: float = 0.0
    shape_erank_reg: float = 0.0
    shape_erank_s3_reg: float = 0.0
    shape_quat_norm_reg: float = 0.0
    capture_opacity_gradient: bool = False
    shape_axis_ratio_reg: float = 0.0
    shape_max_axis_ratio: float = 100.0


@dataclass
class ModelGradients:
    means: Optional[torch.Tensor] = None
    log_scales: Optional[torch.Tensor] = None
    quaternions: Optional[torch.Tensor] = None
    opacity_logits: Optional[torch.Tensor] = None
    sh: Optional[torch.Tensor] = None
    colors_precomp: Optional[torch.Tensor] = None
    refine_weight: Optional[torch.Tensor] = None
    densify_weight: Optional[torch.Tensor] = None
    densify_weight_den: Optional[torch.Tensor] = None


# --------------------------------------------------------------- contexts --
class _Context:
    """One native gs_context (workspace owner). Returned to its pool on release."""

    def __init__(self, pool: "_ContextPool"):
        self.pool = pool
        self.ptr = C.c_void_p()
        lib = L.load()
        L.check(lib.gs_create(C.byref(self.ptr), pool.device, None), None)

    def bind_stream(self) -> None:
        stream = torch.cuda.current_stream(self.pool.device).cuda_stream
        L.check(L.load().gs_set_stream(self.ptr, C.c_void_p(stream)), self.ptr)

    def release(self) -> None:
        self.pool.give_back(self)

    def destroy(self) -> None:
        if self.ptr:
            L.load().gs_destroy(self.ptr)
            self.ptr = C.c_void_p()


class _ContextPool:
    def __init__(self, device: int):
        self.device = device
        self.free: list[_Context] = []
        self.lock = threading.Lock()

    def take(self) -> _Context:
        with self.lock:
            if self.free:
                return self.free.pop()
        return _Context(self)

    def give_back(self, ctx: _Context) -> None:
        with self.lock:
            self.free.append(ctx)


_POOLS: dict[int, _ContextPool] = {}


def _pool(device: int) -> _ContextPool:
    if device not in _POOLS:
        _POOLS[device] = _ContextPool(device)
    return _POOLS[device]


class _Live:
    """Holds a context for the lifetime of a RenderResult."""

    def __init__(self, ctx: _Context, keep: tuple):
        self.ctx = ctx
        self.keep = keep  # tensors the native side reads again in backward
        self.backward_done = False

    def __del__(self):
        try:
            self.ctx.release()
        except Exception:
            pass


@dataclass
class RenderResult:
    color: torch.Tensor
    alpha: torch.Tensor
    radii: torch.Tensor
    visibility: torch.Tensor
    rendered_instances: int = 0
    visible_count: int = 0
    depth_bits: int = 0
    tile_bits: int = 0
    context: Optional[_Live] = None
    median_depth: Optional[torch.Tensor] = None  # [H,W] with require_depth
    normal: Optional[torch.Tensor] = None        # [3,H,W] with require_depth


# ---------------------------------------------------------------- helpers --
def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _require(t: Optional[torch.Tensor], name: str, dtype=torch.float32) -> None:
    if t is None or not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous CUDA {str(dtype).split('.')[-1]} tensor")


def _camera_struct(cam: Camera, policy: RasterizationPolicy) -> L.Camera:
    c = L.Camera()
    c.width, c.height = int(cam.width), int(cam.height)
    c.fx, c.fy = float(cam.fx), float(cam.fy)
    # Integer pixel centres become half-integer samples by shifting the
    # principal point (photara/src/splat/rasterizer.cu:209-212).
    c.cx = float(cam.cx) - policy.pixel_center_offset
    c.cy = float(cam.cy) - policy.pixel_center_offset
    c.near_plane = float(policy.near_plane)
    c.alpha_clip = float(policy.alpha_clip)
    c.compensate_2d = 1 if policy.compensate_2d else 0
    w2c = [float(v) for v in cam.world_to_camera]
    if len(w2c) != 16:
        raise ValueError("world_to_camera must hold 16 floats")
    c.world_to_camera[:] = w2c
    c.center[:] = [float(v) for v in cam.position]
    return c


def look_at_camera(eye, target, up, width, height, fx, fy=None, cx=None, cy=None) -> Camera:
    """Pinhole camera at `eye` looking at `target` (+z forward, +y down in the image)."""
    import numpy as np
    eye = np.asarray(eye, dtype=np.float64)
    f = np.asarray(target, dtype=np.float64) - eye
    f /= np.linalg.norm(f)
    u = np.asarray(up, dtype=np.float64)
    r = np.cross(f, u)
    r /= np.linalg.norm(r)
    d = np.cross(f, r)  # image down
    R = np.stack([r, d, f])  # rows: camera axes in world
    t = -R @ eye
    M = np.eye(4)
    M[:3, :3] = R
    M[:3, 3] = t
    col_major = M.T.reshape(-1).astype(np.float32).tolist()
    return Camera(col_major, eye.astype(np.float32).tolist(), fx, fy if fy is not None else fx,
                  cx if cx is not None else width / 2.0, cy if cy is not None else height / 2.0,
                  int(width), int(height))


# ------------------------------------------------------------- rasterizer --
class Rasterizer:
    """Drop-in for photara::splat::Rasterizer (CUDA 3DGS pinhole RGB path).

    pixels_per_thread selects the compositing schedule (1, 2, 4 or 8; None =
    chosen per frame from its tile count); results do not depend on it."""

    def __init__(self, pixels_per_thread: Optional[int] = None):
        self.pixels_per_thread = pixels_per_thread

    def forward(self, model: GaussianModel, camera: Camera,
                options: Optional[RasterizeOptions] = None) -> RenderResult:
        options = options or RasterizeOptions()
        self._validate_model(model, options)
        if camera.width == 0 or camera.height == 0:
            raise ValueError("Splat camera dimensions must be positive")
        dev = model.means.device
        n = model.size()
        H, W = int(camera.height), int(camera.width)
        color = torch.empty((3, H, W), device=dev, dtype=torch.float32)
        alpha = torch.empty((H, W), device=dev, dtype=torch.float32)
        radii = torch.empty((n,), device=dev, dtype=torch.int32)  # written for every Gaussian
        visibility = torch.zeros((n,), device=dev, dtype=torch.float32)
        result = RenderResult(color, alpha, radii, visibility)
        if options.require_depth:
            result.median_depth = torch.empty((H, W), device=dev, dtype=torch.float32)
            result.normal = torch.empty((3, H, W), device=dev, dtype=torch.float32)
        if n == 0:
            color.copy_(torch.tensor(list(options.background), device=dev).view(3, 1, 1)
                        .expand(3, H, W))
            alpha.zero_()
            if options.require_depth:
                result.median_depth.zero_()
                result.normal.zero_()
            return result
        sh_degree = min(int(options.active_sh_degree), int(model.sh_degree))
        g = L.Gaussians()
        g.count = n
        g.means = _ptr(model.means)
        g.log_scales = _ptr(model.log_scales)
        g.quaternions = _ptr(model.quaternions)
        g.opacity_logits = _ptr(model.opacity_logits)
        g.filter_3d = _ptr(model.filter_3d)
        if options.colors_precomp is not None:
            g.colors = _ptr(options.colors_precomp)
            g.sh, g.sh_degree, g.sh_bases = None, 0, 0
        else:
            g.sh = _ptr(model.sh)
            g.sh_degree = sh_degree
            g.sh_bases = int(model.sh.shape[1])
        s = L.Settings()
        s.background[:] = [float(v) for v in options.background]
        s.scale_modifier = float(options.scale_modifier)
        s.kernel_size = float(options.kernel_size)
        s.record_backward_state = 1 if options.record_backward_state else 0
        s.need_depth = 1 if options.require_depth else 0
        out = L.Outputs(_ptr(color), _ptr(alpha), _ptr(visibility), _ptr(radii),
                        _ptr(result.median_depth), _ptr(result.normal))
        info = L.ForwardInfo()
        ctx = _pool(dev.index if dev.index is not None else torch.cuda.current_device()).take()
        try:
            ctx.bind_stream()
            L.check(L.load().gs_set_schedule(ctx.ptr, int(self.pixels_per_thread or 0)), ctx.ptr)
            L.check(L.load().gs_forward(ctx.ptr, C.byref(g), C.byref(_camera_struct(
                camera, options.rasterization)), C.byref(s), C.byref(out), C.byref(info)), ctx.ptr)
        except Exception:
            ctx.release()
            raise
        keep = (model.means, model.log_scales, model.quaternions, model.opacity_logits, model.sh,
                model.filter_3d, options.colors_precomp)
        result.context = _Live(ctx, keep)
        result.context.options = options
        result.context.model = model
        result.rendered_instances = int(info.instance_count)
        result.visible_count = int(info.visible_count)
        result.depth_bits = int(info.depth_bits)
        result.tile_bits = int(info.tile_bits)
        return result

    def backward(self, model: GaussianModel, rendered: RenderResult, grad_color: torch.Tensor,
                 grad_alpha: Optional[torch.Tensor] = None, grad_depth=None, grad_normal=None,
                 densify_map: Optional[torch.Tensor] = None,
                 sh_adam: Optional[SHAdamUpdate] = None,
                 structure_adam: Optional[StructureAdamUpdate] = None,
                 activated_gradients: bool = False) -> ModelGradients:
        live = rendered.context
        if live is None:
            raise ValueError("Splat backward requires a live forward context")
        options: RasterizeOptions = live.options
        if not options.record_backward_state:
            raise L.StateError(L.GS_ERR_STATE, "Cannot backpropagate an inference-only render")
        _require(grad_color, "grad_color")
        if grad_depth is not None or grad_normal is not None:
            # gradients of the median-depth / normal channels (the reference's
            # GEOMETRY backward); the forward's depth and normal outputs are
            # read again and must be unchanged since the forward
            if not options.require_depth:
                raise L.StateError(L.GS_ERR_STATE, "median-depth / normal gradients need a "
                                   "forward with require_depth")
            H, W = rendered.alpha.shape
            if grad_depth is not None:
                _require(grad_depth, "grad_depth")
                if tuple(grad_depth.shape) != (H, W):
                    raise ValueError("grad_depth must be [H,W]")
            if grad_normal is not None:
                _require(grad_normal, "grad_normal")
                if tuple(grad_normal.shape) != (3, H, W):
                    raise ValueError("grad_normal must be [3,H,W]")
        if grad_alpha is not None:
            _require(grad_alpha, "grad_alpha")
        if densify_map is not None and densify_map.numel() != 0:
            _require(densify_map, "densify_map")
        else:
            densify_map = None
        n = model.size()
        dev = model.means.device
        precomp = options.colors_precomp is not None
        if sh_adam is not None and (precomp or model.sh.shape[1] > 16 or
                                    sh_adam.first.numel() != model.sh.numel() or
                                    sh_adam.first.dtype != torch.float16 or
                                    sh_adam.packed.numel() != model.sh.numel() or
                                    sh_adam.packed.dtype != torch.uint8 or
                                    sh_adam.bounds.numel() != n * 4):
            raise ValueError("Incompatible fused SH Adam context/state")
        if structure_adam is not None and (
                precomp or structure_adam.means_first.numel() != model.means.numel() or
                structure_adam.means_second.numel() != model.means.numel() or
                structure_adam.scales_first.numel() != model.log_scales.numel() or
                structure_adam.scales_second.numel() != model.log_scales.numel() or
                structure_adam.rotations_first.numel() != model.quaternions.numel() or
                structure_adam.rotations_second.numel() != model.quaternions.numel() or
                structure_adam.opacity_first.numel() != model.opacity_logits.numel() or
                structure_adam.opacity_second.numel() != model.opacity_logits.numel()):
            raise ValueError("Incompatible fused structure Adam context/state")
        grads = ModelGradients()
        fuse_structure = structure_adam is not None
        z = lambda *shape: torch.zeros(shape, device=dev, dtype=torch.float32)
        if not fuse_structure:
            grads.means = z(n, 3)
            grads.log_scales = z(n, 3)
            grads.quaternions = z(n, 4)
            grads.opacity_logits = z(n, 1)
        elif structure_adam.capture_opacity_gradient:
            grads.opacity_logits = z(n, 1)
        if sh_adam is None and not precomp:
            grads.sh = torch.zeros_like(model.sh)
        if precomp:
            grads.colors_precomp = z(n, 3)
        grads.refine_weight = z(n)
        if densify_map is not None:
            grads.densify_weight = z(n)
            grads.densify_weight_den = z(n)
        mg = L.ModelGrads()
        if not fuse_structure:
            mg.means = _ptr(grads.means)
            mg.scales = _ptr(grads.log_scales)
            mg.rotations = _ptr(grads.quaternions)
            mg.opacities = _ptr(grads.opacity_logits)
        mg.sh = _ptr(grads.sh)
        mg.colors = _ptr(grads.colors_precomp)
        mg.refine_weight = _ptr(grads.refine_weight)
        mg.densify_weight = _ptr(grads.densify_weight)
        mg.densify_weight_den = _ptr(grads.densify_weight_den)
        mg.activated = 1 if activated_gradients else 0
        dl = L.LossGrads(_ptr(grad_color), _ptr(grad_alpha), _ptr(densify_map),
                         _ptr(grad_depth), _ptr(grad_normal))
        sa_p = None
        if fuse_structure:
            a = structure_adam
            sa = L.StructureAdam()
            sa.means, sa.log_scales = _ptr(model.means), _ptr(model.log_scales)
            sa.quaternions, sa.opacity_logits = _ptr(model.quaternions), _ptr(model.opacity_logits)
            for name in ("means_first", "means_second", "scales_first", "scales_second",
                         "rotations_first", "rotations_second", "opacity_first", "opacity_second"):
                setattr(sa, name, _ptr(getattr(a, name)))
            sa.filter_3d = _ptr(model.filter_3d)
            for name in ("means_lr", "scales_lr", "quaternions_lr", "opacities_lr", "beta1",
                         "beta2", "correction1", "correction2", "epsilon", "opacity_reg",
                         "scale_reg", "shape_erank_reg", "shape_erank_s3_reg",
                         "shape_quat_norm_reg", "shape_axis_ratio_reg", "shape_max_axis_ratio"):
                setattr(sa, name, float(getattr(a, name)))
            sa.minimum_log_scale = max(float(a.minimum_log_scale), -3.0e38)
            sa.maximum_log_scale = min(float(a.maximum_log_scale), 3.0e38)
            sa.opacity_gradient = _ptr(grads.opacity_logits) if a.capture_opacity_gradient else None
            sa_p = C.byref(sa)
        sh_p = None
        if sh_adam is not None:
            stride = int(model.sh.shape[1]) * 3
            reg = (2.0 * sh_adam.regularization_weight / float(n * (stride - 3))
                   if stride > 3 and sh_adam.regularization_weight > 0 else 0.0)
            sh = L.ShAdam()
            sh.parameter = _ptr(model.sh)
            sh.lr, sh.rest_lr = float(sh_adam.lr), float(sh_adam.rest_lr)
            sh.beta1, sh.beta2 = float(sh_adam.beta1), float(sh_adam.beta2)
            sh.correction1, sh.correction2 = float(sh_adam.correction1), float(sh_adam.correction2)
            sh.epsilon = float(sh_adam.epsilon)
            sh.regularization_factor = reg
            sh.first, sh.packed, sh.bounds = (_ptr(sh_adam.first), _ptr(sh_adam.packed),
                                              _ptr(sh_adam.bounds))
            sh.stride = stride
            sh_p = C.byref(sh)
        if n != 0 and rendered.rendered_instances > 0:
            live.ctx.bind_stream()
            L.check(L.load().gs_backward(live.ctx.ptr, _ptr(rendered.alpha), _ptr(rendered.radii),
                                         C.byref(dl), C.byref(mg), sa_p, sh_p), live.ctx.ptr)
        live.backward_done = True
        return grads

    def forward_colors(self, rendered: RenderResult, colors: torch.Tensor) -> RenderResult:
        """Blend new precomputed colours [N,3] over the draw list of a training
        forward that used colors_precomp (splat_drender Rasterizer::forward_colors,
        pipeline.cu:617-649). The forward context moves to the returned result,
        whose backward differentiates this blend."""
        live = rendered.context
        if live is None or not live.options.record_backward_state:
            raise L.StateError(L.GS_ERR_STATE, "color reuse requires a training forward")
        if live.options.colors_precomp is None:
            raise L.StateError(L.GS_ERR_STATE, "color reuse requires precomputed colors")
        _require(colors, "colors")
        n = live.model.size()
        if tuple(colors.shape) != (n, 3):
            raise ValueError("colors must be [N,3]")
        color = torch.empty_like(rendered.color)
        alpha = torch.empty_like(rendered.alpha)
        visibility = torch.zeros_like(rendered.visibility)
        out = L.Outputs(_ptr(color), _ptr(alpha), _ptr(visibility), _ptr(rendered.radii), None,
                        None)
        if n != 0:
            live.ctx.bind_stream()
            L.check(L.load().gs_forward_colors(live.ctx.ptr, _ptr(colors), C.byref(out)),
                    live.ctx.ptr)
        else:
            color.copy_(rendered.color)
            alpha.copy_(rendered.alpha)
        live.options = replace(live.options, colors_precomp=colors)
        live.keep = live.keep + (colors,)
        live.backward_done = False
        result = RenderResult(color, alpha, rendered.radii, visibility,
                              rendered.rendered_instances, rendered.visible_count,
                              rendered.depth_bits, rendered.tile_bits, live)
        rendered.context = None
        return result

    def pruning_scores(self, model: GaussianModel, camera: Camera,
                       options: Optional[RasterizeOptions] = None,
                       gaussian_pop: bool = False) -> torch.Tensor:
        """Speedy-Splat pruning score of every Gaussian for one view
        (CudaRasterizer::pruning_scores, photara/src/splat/rasterizer.cu:450):
        renders `camera` (colour only, per-pixel state recorded) and returns
        the scores [N] (sum over views by adding the results)."""
        options = replace(options or RasterizeOptions(), require_depth=False,
                          record_backward_state=True, colors_precomp=None)
        rendered = self.forward(model, camera, options)
        scores = torch.zeros((model.size(),), device=model.means.device, dtype=torch.float32)
        if model.size() == 0 or rendered.rendered_instances == 0:
            return scores
        live = rendered.context
        live.ctx.bind_stream()
        L.check(L.load().gs_pruning_scores(live.ctx.ptr, _ptr(rendered.color),
                                           1 if gaussian_pop else 0, _ptr(scores)), live.ctx.ptr)
        return scores

    def attribute_error(self, model: GaussianModel, rendered: RenderResult,
                        error_map: torch.Tensor, num: torch.Tensor, den: torch.Tensor) -> None:
        """Adds sum(error * alpha * T) and sum(alpha * T) over the pixels that
        each Gaussian reaches in `rendered` into num / den ([N] float32): the
        densify weights of the backward, with no parameter gradient formed."""
        live = rendered.context
        if live is None or not live.options.record_backward_state:
            raise L.StateError(L.GS_ERR_STATE, "Error attribution needs a backward-ready render")
        _require(error_map, "error_map")
        _require(num, "num")
        _require(den, "den")
        n = model.size()
        if num.numel() != n or den.numel() != n or error_map.numel() != rendered.alpha.numel():
            raise ValueError("error attribution buffers do not match the render")
        zero = torch.zeros_like(rendered.color)
        mg = L.ModelGrads()
        mg.densify_weight, mg.densify_weight_den = _ptr(num), _ptr(den)
        dl = L.LossGrads(_ptr(zero), None, _ptr(error_map))
        if n != 0 and rendered.rendered_instances > 0:
            live.ctx.bind_stream()
            L.check(L.load().gs_backward(live.ctx.ptr, _ptr(rendered.alpha), _ptr(rendered.radii),
                                         C.byref(dl), C.byref(mg), None, None), live.ctx.ptr)
        live.backward_done = True

    @staticmethod
    def _validate_model(model: GaussianModel, options: RasterizeOptions) -> None:
        for name in ("means", "log_scales", "quaternions", "opacity_logits", "sh"):
            _require(getattr(model, name), f"model.{name}")
        if model.filter_3d is not None:
            _require(model.filter_3d, "model.filter_3d")
        if options.colors_precomp is not None:
            _require(options.colors_precomp, "colors_precomp")
        n = model.size()
        m = model
        bad = (m.means.dim() != 2 or m.means.shape[1] != 3 or m.log_scales.shape != m.means.shape or
               m.quaternions.dim() != 2 or m.quaternions.shape[0] != n or m.quaternions.shape[1] != 4
               or m.opacity_logits.numel() != n or m.sh.dim() != 3 or m.sh.shape[0] != n or
               m.sh.shape[2] != 3 or (m.filter_3d is not None and m.filter_3d.numel() != n))
        if bad:
            raise ValueError("Invalid splat model tensor shapes")
        if options.colors_precomp is not None and tuple(options.colors_precomp.shape) != (n, 3):
            raise ValueError("Precomputed colors must have shape [N,3]")


# ------------------------------------------------------------- debug view --
def draw_list(rendered: RenderResult):
    """(sorted 64-bit keys, Gaussian ids in composite order, tile ranges [T,2])."""
    live = rendered.context
    if live is None:
        raise ValueError("no live forward")
    I = rendered.rendered_instances
    dev = rendered.color.device
    H, W = rendered.alpha.shape
    tiles = ((W + 15) // 16) * ((H + 15) // 16)
    keys = torch.empty((max(I, 1),), dtype=torch.int64, device=dev)
    vals = torch.empty((max(I, 1),), dtype=torch.int32, device=dev)
    ranges = torch.empty((tiles, 2), dtype=torch.int32, device=dev)
    live.ctx.bind_stream()
    L.check(L.load().gs_debug_draw_list(live.ctx.ptr, _ptr(keys), _ptr(vals), _ptr(ranges)),
            live.ctx.ptr)
    return keys[:I], vals[:I], ranges


def stage_times(rendered: RenderResult) -> list[float]:
    live = rendered.context
    buf = (C.c_float * 8)()
    L.check(L.load().gs_stage_times(live.ctx.ptr, buf, 8), live.ctx.ptr)
    return list(buf)
