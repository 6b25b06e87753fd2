"""Bounded device-side waits: a look-back wait whose predecessor is never
published gives up after its limit, the kernel returns, and the host reports
GS_ERR_TIMEOUT with the context still usable.

The reference's CUB sorts have no such wait; these waits belong to this
library's single-pass scan and onesweep sort, and to the compositing kernels'
staging (an mbarrier phase their TMA gathers complete). The probe
(gs_debug_lookback_probe) runs the production scan kernel, or one onesweep
pass, as a single block that takes tile 1 while tile 0 is never published: a
flag that nothing sets, with the wait limited to a few thousand re-reads; or
one block whose mbarrier expects bytes that no copy delivers. No test here faults, traps or
hangs the GPU: every wait ends by itself and every access stays in bounds.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import camera_of, device_model, gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]

GS_OK, GS_ERR_TIMEOUT = 0, 5


@pytest.fixture()
def ctx():
    c = gsb.rasterizer._pool(0).take()
    c.bind_stream()
    yield c
    c.release()


@pytest.mark.parametrize("which", [0, 1, 2], ids=["scan", "onesweep", "staging"])
def test_unpublished_predecessor_times_out_and_is_reported(ctx, which):
    lib = gsb.load_library()
    assert lib.gs_device_status(ctx.ptr) == GS_OK
    assert lib.gs_debug_lookback_probe(ctx.ptr, which, 4096) == GS_ERR_TIMEOUT
    assert b"timed out" in lib.gs_last_error(ctx.ptr)
    # the word was reported once and cleared: the context is usable again
    assert lib.gs_device_status(ctx.ptr) == GS_OK
    n = 100_003
    src = torch.arange(n, dtype=torch.int32, device="cuda") % 7
    dst = torch.empty_like(src)
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.gs_exclusive_scan_u32(ctx.ptr, src.data_ptr(), dst.data_ptr(), n,
                                     total.data_ptr()) == GS_OK
    assert lib.gs_device_status(ctx.ptr) == GS_OK
    a = src.cpu().numpy().astype(np.int64)
    assert np.array_equal(dst.cpu().numpy(), np.concatenate([[0], np.cumsum(a)[:-1]]))


def test_probe_rejects_limits_outside_its_range(ctx):
    lib = gsb.load_library()
    assert lib.gs_debug_lookback_probe(ctx.ptr, 3, 100) == 1
    assert lib.gs_debug_lookback_probe(ctx.ptr, 0, 0) == 1
    assert lib.gs_debug_lookback_probe(ctx.ptr, 0, (1 << 20) + 1) == 1


def test_rendering_after_a_timeout_is_unaffected():
    """A forward, then a timed-out probe on the context that forward used,
    then the same forward + a backward on that context again: the image is
    identical and the backward runs."""
    scene = gsb.make_scene("small", seed=3)
    model, cam = device_model(scene), camera_of(scene)
    rast = gsb.Rasterizer()
    r0 = rast.forward(model, cam)
    color0 = r0.color.clone()
    del r0  # its context goes back to the pool
    lib = gsb.load_library()
    pool = gsb.rasterizer._pool(0)
    ctx = pool.take()
    ctx.bind_stream()
    assert lib.gs_debug_lookback_probe(ctx.ptr, 1, 2048) == GS_ERR_TIMEOUT
    ctx.release()
    r = rast.forward(model, cam)
    assert r.context.ctx is ctx  # the pool hands the same context back
    g = rast.backward(model, r, torch.full_like(r.color, 1e-3), None)
    torch.cuda.synchronize()
    assert torch.equal(r.color, color0)
    assert torch.isfinite(g.means).all() and g.means.abs().sum() > 0
