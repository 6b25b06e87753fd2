"""Generates the golden fixtures that pin the CPU oracle to the reference.

Runs the reference rasterizer itself (oracle/_ref/libsplat_ref.so, compiled
from the reference's splat_drender sources) on seeded synthetic scenes and
stores its outputs. Needs a CUDA GPU; the fixtures are committed so the CPU
test suite can check the oracle without one.

    python tests/golden/make_golden.py          # writes tests/golden/*.npz

Inputs are not stored: they are regenerated from (scene name, seed) by
make_scene(), and the per-pixel loss gradients by loss_grads() below.
"""
from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

# (scene, seed, background); the SH gradient is stored for the tiny case only
# to keep the fixtures small.
CASES = [("tiny", 0, (0.0, 0.0, 0.0)), ("small", 1, (0.2, 0.1, 0.05))]


def loss_grads(scene, seed):
    rng = np.random.default_rng(1000 + seed)
    gc = (rng.normal(size=(3, scene.height, scene.width)) * 1e-3).astype(np.float32)
    ga = (rng.normal(size=(scene.height, scene.width)) * 1e-3).astype(np.float32)
    return gc, ga


def main():
    import torch
    gsb = importlib.import_module("photara-studio_b200")
    from oracle import reference as ref
    for name, seed, bg in CASES:
        scene = gsb.make_scene(name, seed=seed)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        model = gsb.GaussianModel(t(scene.means), t(scene.log_scales), t(scene.quaternions),
                                  t(scene.opacity_logits), t(scene.sh), 3)
        cam = gsb.Camera(scene.world_to_camera, scene.position, scene.fx, scene.fy, scene.cx,
                         scene.cy, scene.width, scene.height)
        fwd = ref.forward(model, cam, background=bg)
        vals, ranges = ref.draw_list(fwd["instances"], cam.width, cam.height, "cuda")
        gc, ga = loss_grads(scene, seed)
        grads = ref.backward(fwd, t(gc), t(ga), model.size(), model.sh.numel(), "cuda")
        torch.cuda.synchronize()
        out = {"color": fwd["color"], "alpha": fwd["alpha"], "radii": fwd["radii"],
               "visibility": fwd["visibility"], "values": vals, "ranges": ranges}
        out.update({"grad_" + k: v for k, v in grads.items() if k != "sh" or name == "tiny"})
        arrays = {k: v.cpu().numpy() for k, v in out.items()}
        arrays["instances"] = np.int64(fwd["instances"])
        arrays["visible"] = np.int64(fwd["visible"])
        arrays["background"] = np.asarray(bg, np.float32)
        np.savez_compressed(HERE / f"ref_{name}_s{seed}.npz", **arrays)
        print(f"{name}: instances={fwd['instances']} visible={fwd['visible']}")


if __name__ == "__main__":
    main()
