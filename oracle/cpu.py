"""Python driver of the CPU oracle (oracle/splat_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker, never by the product.

The C loops take [begin, end) ranges; host threads run disjoint ranges (ctypes
releases the GIL), each with a private gradient buffer for the compositing
adjoint. Sorting of the 64-bit keys uses numpy's stable argsort.
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import os
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
TILE = 16

_lib = None


class OrcCamera(C.Structure):
    _fields_ = [("view", C.c_float * 16), ("center", C.c_float * 3), ("fx", C.c_float),
                ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("near_plane", C.c_float), ("alpha_clip", C.c_float), ("width", C.c_int),
                ("height", C.c_int), ("compensate_2d", C.c_int), ("kernel_size", C.c_float),
                ("scale_modifier", C.c_float)]


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            import subprocess
            subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
        _lib = C.CDLL(str(LIB))
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def threads() -> int:
    return max(1, min(os.cpu_count() or 1, 32))


def _parallel(fn, total: int, nthreads: int):
    nthreads = max(1, min(nthreads, total))
    bounds = np.linspace(0, total, nthreads + 1).astype(int)
    with cf.ThreadPoolExecutor(max_workers=nthreads) as ex:
        list(ex.map(lambda k: fn(int(bounds[k]), int(bounds[k + 1]), k), range(nthreads)))


def camera(scene, kernel_size=0.0, compensate_2d=True, near_plane=0.2, alpha_clip=0.99,
           scale_modifier=1.0) -> OrcCamera:
    c = OrcCamera()
    c.view[:] = [float(v) for v in scene.world_to_camera]
    c.center[:] = [float(v) for v in scene.position]
    c.fx, c.fy, c.cx, c.cy = scene.fx, scene.fy, scene.cx, scene.cy
    c.near_plane, c.alpha_clip = near_plane, alpha_clip
    c.width, c.height = scene.width, scene.height
    c.compensate_2d = 1 if compensate_2d else 0
    c.kernel_size, c.scale_modifier = kernel_size, scale_modifier
    return c


def crop_tiles(scene, x0: int, y0: int, w: int, h: int) -> list:
    """Tile-index ranges [begin, end) covering the pixel crop (x0, y0, w, h),
    one range per tile row."""
    gx = (scene.width + TILE - 1) // TILE
    tx0, tx1 = x0 // TILE, (x0 + w + TILE - 1) // TILE
    return [(ty * gx + tx0, ty * gx + tx1) for ty in range(y0 // TILE, (y0 + h + TILE - 1) // TILE)]


def render(scene, background=(0.0, 0.0, 0.0), kernel_size=0.0, sh_degree=3, use_double=True,
           nthreads: int | None = None, means=None, tile_subset=None) -> dict:
    """Oracle forward. Returns images (float64), per-Gaussian state and the draw list.
    tile_subset: optional [begin, end) tile ranges; only those tiles are composited
    (the rest of the image stays zero)."""
    lib = load()
    nthreads = nthreads or threads()
    n = scene.count
    cam = camera(scene, kernel_size=kernel_size)
    means = np.ascontiguousarray(scene.means if means is None else means, np.float32)
    ls = np.ascontiguousarray(scene.log_scales, np.float32)
    q = np.ascontiguousarray(scene.quaternions, np.float32)
    lo = np.ascontiguousarray(scene.opacity_logits.reshape(-1), np.float32)
    sh = np.ascontiguousarray(scene.sh, np.float32)
    mean2d = np.zeros((n, 2), np.float32)
    conic = np.zeros((n, 4), np.float32)
    rgb = np.zeros((n, 3), np.float32)
    clamp = np.zeros(n, np.uint8)
    depth = np.zeros(n, np.float32)
    radii = np.zeros(n, np.int32)
    touched = np.zeros(n, np.uint32)
    bounds = np.zeros((n, 4), np.int32)
    _parallel(lambda b, e, k: lib.orc_preprocess(
        n, _p(means), _p(ls), _p(q), _p(lo), _p(sh), sh_degree, sh.shape[1], C.byref(cam),
        _p(mean2d), _p(conic), _p(rgb), _p(clamp), _p(depth), _p(radii), _p(touched),
        _p(bounds), b, e), n, nthreads)
    offsets = np.zeros(n, np.uint64)
    np.cumsum(touched[:-1], out=offsets[1:]) if n > 1 else None
    total = int(touched.sum())
    gx = (scene.width + TILE - 1) // TILE
    gy = (scene.height + TILE - 1) // TILE
    keys = np.zeros(max(total, 1), np.uint64)
    vals = np.zeros(max(total, 1), np.uint32)
    lib.orc_emit(n, _p(mean2d), _p(conic), _p(depth), _p(touched), _p(offsets), gx, gy,
                 _p(keys), _p(vals))
    keys, vals = keys[:total], vals[:total]
    perm = np.argsort(keys, kind="stable")
    keys, vals = keys[perm], vals[perm]
    tiles = gx * gy
    tile_of = (keys >> np.uint64(32)).astype(np.int64)
    starts = np.searchsorted(tile_of, np.arange(tiles), side="left")
    ends = np.searchsorted(tile_of, np.arange(tiles), side="right")
    ranges = np.stack([starts, ends], axis=1).astype(np.uint32)
    ranges[starts == ends] = 0
    P = scene.width * scene.height
    color = np.zeros(3 * P, np.float64)
    alpha = np.zeros(P, np.float64)
    T = np.zeros(P, np.float64)
    last = np.zeros(P, np.uint32)
    vis = np.zeros(n, np.float32)
    bg = np.asarray(background, np.float32)
    comp = lambda b, e, k: lib.orc_composite(
        tiles, _p(ranges), _p(vals), _p(mean2d), _p(conic), _p(rgb), C.byref(cam), _p(bg),
        1 if use_double else 0, _p(color), _p(alpha), _p(T), _p(last), _p(vis), b, e)
    if tile_subset is None:
        _parallel(comp, tiles, nthreads)
    else:
        for k, (b, e) in enumerate(tile_subset):
            comp(b, e, k)
    return {"color": color.reshape(3, scene.height, scene.width),
            "alpha": alpha.reshape(scene.height, scene.width), "T": T, "last": last,
            "visibility": vis, "radii": radii, "touched": touched, "keys": keys,
            "values": vals, "ranges": ranges, "mean2d": mean2d, "conic": conic, "rgb": rgb,
            "clamp": clamp, "depth": depth, "bounds": bounds, "cam": cam, "bg": bg,
            "means": means, "tiles": tiles, "instances": total,
            "visible": int((touched > 0).sum()), "tile_subset": tile_subset}


def geometry(scene, fwd: dict, nthreads: int | None = None) -> dict:
    """Oracle median-depth [H,W] (camera-space Z) and normal [3,H,W] channels
    for the draw list of `fwd` (FP32, the reference's blend_tile<GEOMETRY>)."""
    lib = load()
    nthreads = nthreads or threads()
    n = scene.count
    ls = np.ascontiguousarray(scene.log_scales, np.float32)
    q = np.ascontiguousarray(scene.quaternions, np.float32)
    lo = np.ascontiguousarray(scene.opacity_logits.reshape(-1), np.float32)
    plane = np.zeros((n, 4), np.float32)
    normal = np.zeros((n, 3), np.float32)
    cam = fwd["cam"]
    _parallel(lambda b, e, k: lib.orc_geometry(
        n, _p(fwd["means"]), _p(ls), _p(q), _p(lo), C.byref(cam), _p(fwd["radii"]),
        _p(plane), _p(normal), b, e), n, nthreads)
    P = scene.width * scene.height
    depth = np.zeros(P, np.float32)
    nrm = np.zeros(3 * P, np.float32)
    tiles = fwd["tiles"]
    call = lambda b, e, k: lib.orc_median_depth(
        tiles, _p(fwd["ranges"]), _p(fwd["values"]), _p(fwd["mean2d"]), _p(fwd["conic"]),
        _p(plane), _p(normal), C.byref(cam), _p(depth), _p(nrm), b, e)
    if fwd.get("tile_subset") is None:
        _parallel(call, tiles, nthreads)
    else:
        for k, (b, e) in enumerate(fwd["tile_subset"]):
            call(b, e, k)
    return {"median_depth": depth.reshape(scene.height, scene.width),
            "normal": nrm.reshape(3, scene.height, scene.width), "plane": plane,
            "gaussian_normal": normal}


def backward(scene, fwd: dict, dL_color, dL_alpha=None, activated=False, sh_degree=3,
             nthreads: int | None = None) -> dict:
    """Oracle backward (float64 accumulation). Returns per-parameter gradients."""
    lib = load()
    nthreads = nthreads or threads()
    n = scene.count
    dLc = np.ascontiguousarray(dL_color, np.float32).reshape(-1)
    dLa = None if dL_alpha is None else np.ascontiguousarray(dL_alpha, np.float32).reshape(-1)
    tiles = fwd["tiles"]
    subset = fwd.get("tile_subset")
    k_threads = max(1, min(nthreads, tiles)) if subset is None else 1
    bufs = [np.zeros(12 * n, np.float64) for _ in range(k_threads)]
    call = lambda b, e, k: lib.orc_composite_backward(
        tiles, _p(fwd["ranges"]), _p(fwd["values"]), _p(fwd["mean2d"]), _p(fwd["conic"]),
        _p(fwd["rgb"]), C.byref(fwd["cam"]), _p(fwd["bg"]), _p(fwd["T"]), _p(fwd["last"]),
        _p(dLc), None if dLa is None else _p(dLa), n, _p(bufs[k]), b, e)
    if subset is None:
        _parallel(call, tiles, k_threads)
    else:  # a crop: few tiles, one accumulation buffer
        for b, e in subset:
            call(b, e, 0)
    grad12 = np.sum(bufs, axis=0)
    out = {"means": np.zeros((n, 3)), "scales": np.zeros((n, 3)), "rotations": np.zeros((n, 4)),
           "opacities": np.zeros(n), "sh": np.zeros(scene.sh.shape)}
    means = fwd["means"]
    ls = np.ascontiguousarray(scene.log_scales, np.float32)
    q = np.ascontiguousarray(scene.quaternions, np.float32)
    lo = np.ascontiguousarray(scene.opacity_logits.reshape(-1), np.float32)
    sh = np.ascontiguousarray(scene.sh, np.float32)
    _parallel(lambda b, e, k: lib.orc_gaussian_backward(
        n, _p(means), _p(ls), _p(q), _p(lo), _p(sh), sh_degree, sh.shape[1],
        C.byref(fwd["cam"]), _p(fwd["radii"]), _p(fwd["clamp"]), _p(grad12),
        1 if activated else 0, _p(out["means"]), _p(out["scales"]), _p(out["rotations"]),
        _p(out["opacities"]), _p(out["sh"]), b, e), n, nthreads)
    out["refine_weight"] = grad12.reshape(n, 12)[:, 6].copy()
    out["grad12"] = grad12.reshape(n, 12)
    return out


def adam(param, grad, m, v, lr, b1, b2, c1, c2, eps, lo=-3.0e38, hi=3.0e38):
    """In-place oracle Adam on float32 numpy arrays."""
    lib = load()
    lib.orc_adam(_p(param), _p(grad), _p(m), _p(v), C.c_long(param.size), C.c_float(lr),
                 C.c_float(b1), C.c_float(b2), C.c_float(c1), C.c_float(c2), C.c_float(eps),
                 C.c_float(lo), C.c_float(hi))


def sh_adam_rows(param, grad, first_u16, packed, bounds, active, lr, rest_lr, b1, b2, c1, c2,
                 eps, reg=0.0):
    """In-place oracle quantized SH Adam on rows of float32 / uint16 (fp16 bits) / uint8."""
    lib = load()
    rows, stride = param.shape
    f = C.c_float
    lib.orc_sh_adam_rows(rows, stride, active, _p(param), _p(grad), _p(first_u16), _p(packed),
                         _p(bounds), f(lr), f(rest_lr), f(b1), f(b2), f(c1), f(c2), f(eps),
                         f(reg))


def time_training_step(scene_seed: int = 0, budget_s: float = 20.0) -> dict:
    """CPU baseline: the oracle's forward + backward on the 1080p / 1M-Gaussian
    workload shape, timed on the host cores over a bounded sample (a fraction of
    the Gaussians, rendered into the full 1920x1080 view), scaled to ms/iter of
    the full workload by the Gaussian fraction."""
    import importlib
    import sys
    sys.path.insert(0, str(HERE.parent))
    gsb = importlib.import_module("photara-studio_b200")
    full = gsb.make_scene("g1m_1080p", seed=scene_seed)
    frac_n = 65536
    sub = gsb.make_scene("g1m_1080p", seed=scene_seed, count=frac_n)
    nthreads = threads()
    t0 = time.perf_counter()
    reps = 0
    while True:
        fwd = render(sub, nthreads=nthreads, use_double=False)
        g = np.full((3, sub.height, sub.width), 1e-6, np.float32)
        backward(sub, fwd, g, nthreads=nthreads)
        reps += 1
        if time.perf_counter() - t0 > budget_s or reps >= 3:
            break
    sec = (time.perf_counter() - t0) / reps
    scale = full.count / frac_n
    return {"value": round(sec * scale * 1e3, 1), "unit": "ms/iter", "cores": nthreads,
            "kind": "port",
            "sample": f"{frac_n} of {full.count} Gaussians at 1920x1080, forward+backward, "
                      f"{reps} rep(s), time scaled by the Gaussian fraction ({scale:.0f}x)"}
