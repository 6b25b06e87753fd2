"""Builds the sm_100a shared library libgsplat_b200.so in-tree with nvcc.

The library is a plain C ABI (include/gsplat_b200.h) with no torch types, so it
is compiled directly with nvcc rather than as a torch extension. Objects go to
`_build/`; the .so lands next to this file so it travels with the package.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libgsplat_b200.so"
SOURCES = ["preprocess.cu", "sort_scan.cu", "composite.cu", "gaussian_backward.cu", "ssim.cu",
           "image_loss.cu", "capi.cu", "noalloc.cu", "densify.cu", "densify_apply.cu", "mlp.cu",
           "batch.cu", "prune_scores.cu", "forward_colors.cu"]

# Same floating-point semantics as the reference's build (-use_fast_math:
# FTZ, approximate division/sqrt, contraction), required for bit-exact keys.
NVCC_FLAGS = [
    "-O3", "-std=c++20", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-use_fast_math", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden",
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found")
    return exe


def _compile(src: Path, obj: Path, extra: list[str]) -> None:
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
    if res.stderr.strip() and os.environ.get("GSB_VERBOSE"):
        sys.stderr.write(res.stderr)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [
        HERE.parent / "include" / "gsplat_b200.h"]
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    jobs = []
    objs = []
    for name in SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        objs.append(obj)
        if force or verbose_ptxas or _stale(obj, [src, *headers]):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for f in [ex.submit(_compile, s, o, extra) for s, o in jobs]:
                f.result()
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o",
               str(LIB) + ".tmp", *map(str, objs), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
        os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv))
