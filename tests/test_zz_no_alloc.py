"""The allocation-free scan, gs_exclusive_scan_u32_noalloc.

Some callers cannot allocate device memory at the point where they need a
scan: cudaMalloc synchronises the whole device (a stall inside a real-time
render or training loop), and it is off limits to plugins whose host
application owns every device allocation. For them the library keeps the
scan's scratch in a fixed device array and this entry point takes only the
input and output buffers.

This file is collected last so that a run stopping at its first failure has
already run every other test. Each check goes through the C ABI and compares
the allocation-free scan with gs_exclusive_scan_u32, the regular entry point
whose scratch lives in a context; integer results must be identical.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]

MAX_ELEMENTS = 33_554_432  # the scratch array's capacity (2^25 elements)
GS_ERR_CAPACITY = 4


def _regular_scan(lib, ctx, src):
    out = torch.empty_like(src)
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.gs_exclusive_scan_u32(ctx.ptr, src.data_ptr(), out.data_ptr(), src.numel(),
                                     total.data_ptr()) == 0
    return out, total


def _noalloc_scan(lib, src, status=None):
    out = torch.full_like(src, -1)
    total = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.gs_exclusive_scan_u32_noalloc(src.data_ptr(), out.data_ptr(), src.numel(),
                                             total.data_ptr(), stream) == 0
    if status is not None:
        # the scan's error word, copied into a caller-owned device word
        assert lib.gs_exclusive_scan_u32_noalloc_status(status.data_ptr(), stream) == 0
    return out, total


def test_noalloc_scan_matches_regular_scan_on_two_calls_in_a_row():
    lib = gsb.load_library()
    ctx = gsb.rasterizer._pool(0).take()
    ctx.bind_stream()
    try:
        rng = np.random.default_rng(42)
        status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        # Two calls in a row on the shared scratch: a large one, then a smaller
        # one that must not see the first call's look-back state.
        for n in (3_000_000, 1_234_567):
            a = rng.integers(0, 64, size=n, dtype=np.int32)
            src = torch.from_numpy(a).cuda()
            ref_out, ref_total = _regular_scan(lib, ctx, src)
            out, total = _noalloc_scan(lib, src, status)
            torch.cuda.synchronize()
            assert torch.equal(out, ref_out)
            assert int(total.item()) == int(ref_total.item()) == int(a.sum())
            assert int(status.item()) == 0  # every look-back wait completed
    finally:
        ctx.release()


def test_noalloc_scan_allocates_nothing_after_its_first_call():
    lib = gsb.load_library()
    src = torch.ones(2_000_000, dtype=torch.int32, device="cuda")
    _noalloc_scan(lib, src)  # first call on the device: one-time address look-up
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    out, total = _noalloc_scan(lib, src)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    assert int(total.item()) == 2_000_000 and int(out[-1].item()) == 1_999_999


def test_noalloc_scan_rejects_sizes_beyond_its_scratch():
    lib = gsb.load_library()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # Rejected on the host before anything is enqueued; the buffers are never touched.
    dummy = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.gs_exclusive_scan_u32_noalloc(dummy.data_ptr(), dummy.data_ptr(),
                                             MAX_ELEMENTS + 1, None, stream) == GS_ERR_CAPACITY
