"""GPU tests of the device-wide scan and onesweep radix sort through the C ABI,
against numpy (bit-exact: integer work)."""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]


@pytest.fixture()
def ctx():
    c = gsb.rasterizer._pool(0).take()
    c.bind_stream()
    yield c
    c.release()


@pytest.mark.parametrize("n", [0, 1, 7, 2047, 2048, 2049, 100_003, 5_000_000])
def test_exclusive_scan_matches_numpy(ctx, n):
    lib = gsb.load_library()
    rng = np.random.default_rng(n)
    a = rng.integers(0, 50, size=n, dtype=np.uint32)
    src = torch.from_numpy(a.view(np.int32)).cuda()
    dst = torch.empty_like(src)
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.gs_exclusive_scan_u32(ctx.ptr, src.data_ptr(), dst.data_ptr(), n,
                                     total.data_ptr()) == 0
    torch.cuda.synchronize()
    expect = np.concatenate([[0], np.cumsum(a, dtype=np.uint64)[:-1]]).astype(np.uint32) if n \
        else np.zeros(0, np.uint32)
    assert np.array_equal(dst.cpu().numpy().view(np.uint32), expect)
    assert int(total.item()) == int(a.sum(dtype=np.uint64))


@pytest.mark.parametrize("n,lo,hi", [(1, 0, 64), (3000, 0, 64), (70_000, 32, 45),
                                     (2_000_000, 0, 40), (4_000_000, 32, 45)])
def test_radix_sort_is_stable_and_exact(ctx, n, lo, hi):
    lib = gsb.load_library()
    rng = np.random.default_rng(n + lo)
    keys = rng.integers(0, 2**63, size=n, dtype=np.uint64)
    dup = keys[::7].copy()
    keys[1::7] = dup[: len(keys[1::7])]  # duplicates to exercise stability
    vals = np.arange(n, dtype=np.uint32)
    kin = torch.from_numpy(keys.view(np.int64)).cuda()
    vin = torch.from_numpy(vals.view(np.int32)).cuda()
    kout, vout = torch.empty_like(kin), torch.empty_like(vin)
    assert lib.gs_sort_pairs_u64(ctx.ptr, kin.data_ptr(), vin.data_ptr(), kout.data_ptr(),
                                 vout.data_ptr(), n, lo, hi) == 0
    torch.cuda.synchronize()
    mask = np.uint64(((1 << (hi - lo)) - 1) if hi - lo < 64 else 2**64 - 1)
    digit = (keys >> np.uint64(lo)) & mask
    perm = np.argsort(digit, kind="stable")
    assert np.array_equal(vout.cpu().numpy().view(np.uint32), vals[perm])
    assert np.array_equal(kout.cpu().numpy().view(np.uint64), keys[perm])
    assert np.array_equal(kin.cpu().numpy().view(np.uint64), keys)  # input untouched


@pytest.mark.parametrize("pixels,offset", [(1, 0), (5, 0), (1920 * 1080, 0), (1001, 1)])
def test_l1_loss_matches_torch(ctx, pixels, offset):
    """gs_l1_loss (photara/src/splat/cuda_ops.cu:1336): grad = w/(3P) sign(d),
    loss += w/(3P) sum |d|; vectorised and scalar (unaligned) paths."""
    lib = gsb.load_library()
    g = torch.Generator(device="cuda").manual_seed(pixels)
    n = 3 * pixels
    img = torch.rand(n + offset, device="cuda", generator=g)[offset:]
    tgt = torch.rand(n + offset, device="cuda", generator=g)[offset:]
    tgt[: n // 7] = img[: n // 7]  # exact zeros of the difference
    grad = torch.empty(n + offset, device="cuda")[offset:]
    loss = torch.zeros(1, device="cuda")
    w = 0.8
    rc = lib.gs_l1_loss(ctx.ptr, img.data_ptr(), tgt.data_ptr(), pixels, w, grad.data_ptr(),
                        loss.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    d = img - tgt
    scale = float(np.float32(w) / np.float32(n))  # the library divides in float32
    assert torch.equal(grad, torch.sign(d) * scale)
    ref = float(d.double().abs().sum()) * scale
    assert abs(float(loss) - ref) <= 1e-5 * max(ref, 1e-6)
