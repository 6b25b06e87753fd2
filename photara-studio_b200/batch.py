"""Batched multi-view rendering and its adjoint (gs_batch_* of the C ABI).

Many cameras of uneven resolution are rendered together: every stage is one
launch over all views, one persistent compositing launch covers the tiles of
every view, and after planning nothing allocates or synchronises, so a whole
forward + backward is captured into one CUDA graph and replayed. Per view the
images equal those of Rasterizer.forward on that camera; gradients are the
sums over views of Rasterizer.backward. The tile shape (8x8, 16x16, 16x32),
pixels per thread and tile schedule are planned explicitly or chosen by the
library's autotuner (schedule="auto").

This replaces a host loop of the reference's one-view-per-call path
(photara/src/splat/rasterizer.cu:390 forward, :681 backward).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence, Union

import torch

from . import _lib as L
from .rasterizer import (Camera, GaussianModel, ModelGradients, RasterizeOptions, _camera_struct,
                         _ptr, _require)

SCHEDULES = {"static": 0, "dynamic": 1, "heavy_first": 2}
_SCHEDULE_NAMES = {v: k for k, v in SCHEDULES.items()}


@dataclass
class BatchSchedule:
    tile_w: int = 16
    tile_h: int = 16
    pixels_per_thread: int = 4
    schedule: str = "dynamic"   # static | dynamic | heavy_first
    ctas_per_sm: int = 0        # 0: as many as fit

    def struct(self) -> L.BatchSchedule:
        return L.BatchSchedule(self.tile_w, self.tile_h, self.pixels_per_thread,
                               SCHEDULES[self.schedule], self.ctas_per_sm)

    @staticmethod
    def of(s: L.BatchSchedule) -> "BatchSchedule":
        return BatchSchedule(s.tile_w, s.tile_h, s.pixels_per_thread,
                             _SCHEDULE_NAMES[s.schedule], s.ctas_per_sm)


@dataclass
class BatchResult:
    color: torch.Tensor      # all views, concatenated planar images
    alpha: torch.Tensor
    radii: torch.Tensor      # [views, N]
    views: list              # (width, height, pixel offset) per view

    def view_color(self, v: int) -> torch.Tensor:
        w, h, off = self.views[v]
        return self.color[3 * off:3 * (off + w * h)].view(3, h, w)

    def view_alpha(self, v: int) -> torch.Tensor:
        w, h, off = self.views[v]
        return self.alpha[off:off + w * h].view(h, w)


class BatchRasterizer:
    """Plans, renders and differentiates one model over many cameras."""

    def __init__(self, device: Optional[int] = None):
        self.device = torch.device("cuda", device if device is not None
                                   else torch.cuda.current_device())
        self.stream = torch.cuda.Stream(device=self.device)
        self._lib = L.load()
        h = C.c_void_p()
        L.check(self._lib.gs_batch_create(C.byref(h), self.device.index,
                                          C.c_void_p(self.stream.cuda_stream)), None)
        self._h = h
        self.schedule: Optional[BatchSchedule] = None
        self.tuning: list = []
        self._keep = ()
        self.result: Optional[BatchResult] = None
        self.grads: Optional[ModelGradients] = None
        self._captured = False

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.gs_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def _check(self, status: int) -> None:
        L.check(status, self._h, batch=True)

    def _enter(self):
        self.stream.wait_stream(torch.cuda.current_stream(self.device))

    def _leave(self):
        torch.cuda.current_stream(self.device).wait_stream(self.stream)

    # ------------------------------------------------------------ planning --
    def plan(self, model: GaussianModel, cameras: Sequence[Camera],
             options: Optional[RasterizeOptions] = None,
             schedule: Union[BatchSchedule, str, None] = None, instance_capacity: int = 0,
             tune_iterations: int = 3) -> "BatchRasterizer":
        options = options or RasterizeOptions(active_sh_degree=model.sh_degree)
        if options.colors_precomp is not None:
            raise ValueError("batched rendering takes SH colours")
        for name in ("means", "log_scales", "quaternions", "opacity_logits", "sh"):
            _require(getattr(model, name), f"model.{name}")
        n = model.size()
        if n == 0 or not cameras:
            raise ValueError("batched rendering needs Gaussians and at least one camera")
        g = L.Gaussians()
        g.count = n
        g.means, g.log_scales = _ptr(model.means), _ptr(model.log_scales)
        g.quaternions, g.opacity_logits = _ptr(model.quaternions), _ptr(model.opacity_logits)
        g.filter_3d = _ptr(model.filter_3d)
        g.sh = _ptr(model.sh)
        g.sh_degree = min(int(options.active_sh_degree), int(model.sh_degree))
        g.sh_bases = int(model.sh.shape[1])
        cams = (L.Camera * len(cameras))(*[_camera_struct(c, options.rasterization)
                                           for c in cameras])
        s = L.Settings()
        s.background[:] = [float(v) for v in options.background]
        s.scale_modifier = float(options.scale_modifier)
        s.kernel_size = float(options.kernel_size)
        s.record_backward_state = 1
        self._enter()
        if schedule == "auto":
            best = L.BatchSchedule()
            best_ms = C.c_float()
            tried = (L.BatchSchedule * 32)()
            tried_ms = (C.c_float * 32)()
            count = C.c_int(32)
            self._check(self._lib.gs_batch_autotune(
                self._h, C.byref(g), cams, len(cameras), C.byref(s), int(tune_iterations),
                C.byref(best), C.byref(best_ms), tried, tried_ms, C.byref(count)))
            self.schedule = BatchSchedule.of(best)
            self.tuning = [(BatchSchedule.of(tried[k]), float(tried_ms[k]))
                           for k in range(count.value)]
            if instance_capacity:
                sc = self.schedule.struct()
                self._check(self._lib.gs_batch_plan(self._h, C.byref(g), cams, len(cameras),
                                                    C.byref(s), C.byref(sc),
                                                    int(instance_capacity)))
        else:
            self.schedule = schedule if isinstance(schedule, BatchSchedule) else BatchSchedule()
            sc = self.schedule.struct()
            self._check(self._lib.gs_batch_plan(self._h, C.byref(g), cams, len(cameras),
                                                C.byref(s), C.byref(sc), int(instance_capacity)))
        self._leave()
        self._keep = (model.means, model.log_scales, model.quaternions, model.opacity_logits,
                      model.sh, model.filter_3d)
        self.model = model
        views, off = [], 0
        for c in cameras:
            views.append((int(c.width), int(c.height), off))
            off += int(c.width) * int(c.height)
        dev = self.device
        self.result = BatchResult(torch.empty(3 * off, device=dev), torch.empty(off, device=dev),
                                  torch.zeros((len(cameras), n), dtype=torch.int32, device=dev),
                                  views)
        self.grads = None
        self._captured = False
        return self

    def info(self) -> dict:
        i = L.BatchInfo()
        self._check(self._lib.gs_batch_get_info(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in L.BatchInfo._fields_}

    # ------------------------------------------------------------ stepping --
    def forward(self) -> BatchResult:
        r = self.result
        self._enter()
        self._check(self._lib.gs_batch_forward(self._h, _ptr(r.color), _ptr(r.alpha),
                                               _ptr(r.radii)))
        self._leave()
        return r

    def _grad_buffers(self) -> ModelGradients:
        m = self.model
        z = torch.zeros_like
        g = ModelGradients(means=z(m.means), log_scales=z(m.log_scales),
                           quaternions=z(m.quaternions), opacity_logits=z(m.opacity_logits),
                           sh=z(m.sh), refine_weight=torch.zeros(m.size(), device=self.device))
        return g

    @staticmethod
    def _model_grads(g: ModelGradients) -> L.ModelGrads:
        mg = L.ModelGrads()
        mg.means, mg.scales = _ptr(g.means), _ptr(g.log_scales)
        mg.rotations, mg.opacities = _ptr(g.quaternions), _ptr(g.opacity_logits)
        mg.sh, mg.refine_weight = _ptr(g.sh), _ptr(g.refine_weight)
        mg.activated = 0
        return mg

    def backward(self, grad_color: torch.Tensor,
                 grad_alpha: Optional[torch.Tensor] = None) -> ModelGradients:
        """Gradients (summed over views) of the last forward; grad_color and
        grad_alpha have the concatenated layout of BatchResult."""
        _require(grad_color, "grad_color")
        if grad_color.numel() != self.result.color.numel():
            raise ValueError("grad_color must match the batched colour layout")
        if grad_alpha is not None:
            _require(grad_alpha, "grad_alpha")
        g = self._grad_buffers()
        self._enter()
        self._check(self._lib.gs_batch_backward(self._h, _ptr(grad_color), _ptr(grad_alpha),
                                                C.byref(self._model_grads(g))))
        self._leave()
        return g

    def capture(self, grad_color: Optional[torch.Tensor] = None,
                grad_alpha: Optional[torch.Tensor] = None) -> None:
        """Captures forward (+ backward into self.grads when grad_color is
        given) into a CUDA graph over the planned buffers."""
        r = self.result
        mg = None
        if grad_color is not None:
            _require(grad_color, "grad_color")
            self.grads = self._grad_buffers()
            mg = C.byref(self._model_grads(self.grads))
            self._capture_inputs = (grad_color, grad_alpha)
        self._enter()
        self._check(self._lib.gs_batch_capture(self._h, _ptr(r.color), _ptr(r.alpha),
                                               _ptr(r.radii), _ptr(grad_color),
                                               _ptr(grad_alpha), mg))
        self._leave()
        self._captured = True

    def replay(self) -> BatchResult:
        """Launches the captured graph; gradients are re-zeroed first (the
        backward accumulates)."""
        if not self._captured:
            raise L.StateError(L.GS_ERR_STATE, "no captured batch graph")
        self._enter()
        with torch.cuda.stream(self.stream):
            if self.grads is not None:
                for t in (self.grads.means, self.grads.log_scales, self.grads.quaternions,
                          self.grads.opacity_logits, self.grads.sh, self.grads.refine_weight):
                    t.zero_()
        self._check(self._lib.gs_batch_replay(self._h))
        self._leave()
        return self.result
