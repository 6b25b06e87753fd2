"""The hand-written adjoint through torch.autograd: gradcheck on smooth scalar
losses of large overlapping Gaussians (the alpha >= 1/255 cut-off is a
discontinuity the adjoint ignores, as the reference's does, so the scene keeps
it a small share of every gradient), and agreement with the CPU oracle."""
import numpy as np
import pytest
import torch

from helpers import gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]


def _params():
    t = lambda a: torch.tensor(a, dtype=torch.float32, device="cuda")
    means = t([[-0.2, 0.1, 3.0], [0.25, -0.05, 3.4], [0.0, 0.3, 3.8]])
    log_scales = torch.log(t([[0.35, 0.2, 0.3], [0.25, 0.4, 0.2], [0.3, 0.3, 0.15]]))
    q = t([[0.9, 0.2, -0.3, 0.1], [0.7, -0.4, 0.2, 0.5], [0.95, 0.1, 0.1, -0.2]])
    quats = q / q.norm(dim=1, keepdim=True)
    logits = t([[0.5], [1.2], [-0.3]])
    g = torch.Generator().manual_seed(0)
    sh = (torch.randn((3, 16, 3), generator=g) * 0.1).cuda()
    sh[:, 0] = t([[0.4, 0.2, 0.1], [0.1, 0.5, 0.2], [0.3, 0.1, 0.4]])
    ident = [1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0]
    cam = gsb.Camera(ident, [0, 0, 0], 64.0, 64.0, 32.0, 24.0, 64, 48)
    return [means, log_scales, quats, logits, sh], cam


def _weights(cam):
    yy, xx = torch.meshgrid(torch.arange(cam.height, dtype=torch.float32),
                            torch.arange(cam.width, dtype=torch.float32), indexing="ij")
    w = torch.stack([1.0 + 0.5 * torch.sin(xx / 9.0), 0.8 + 0.4 * torch.cos(yy / 7.0),
                     0.6 + 0.3 * torch.sin((xx + yy) / 11.0)]).cuda()
    u = (0.3 * torch.cos(xx / 13.0) * torch.sin(yy / 10.0)).cuda()
    return w, u


def test_autograd_gradcheck_on_every_raw_parameter():
    params, cam = _params()
    w, u = _weights(cam)
    opts = gsb.RasterizeOptions(active_sh_degree=3)
    for k in range(5):  # one parameter group at a time keeps the Jacobian small
        def loss(x, k=k):
            ps = [p if i != k else x for i, p in enumerate(params)]
            color, alpha, _ = gsb.rasterize_gaussians(*ps, cam, opts)
            return ((color.double() * w).sum() + (alpha.double() * u).sum()).view(1)
        x = params[k].clone().requires_grad_(True)
        g = torch.autograd.grad(loss(x), x)[0]
        gmax = float(g.abs().max())
        # eps 2e-4: a 1e-3 step of a mean already crosses a discrete footprint
        # event of this scene (the forward is piecewise smooth), while 2e-4
        # stays inside one smooth piece (the CPU oracle shows the same).
        assert torch.autograd.gradcheck(loss, (x,), eps=2e-4, atol=0.01 * gmax, rtol=0.03,
                                        nondet_tol=1e-6 * gmax, raise_exception=True)


def test_autograd_matches_cpu_oracle_raw_gradients():
    cpu = pytest.importorskip("oracle.cpu")
    scene = gsb.make_scene("small", seed=9)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda().requires_grad_(True)
    ps = [t(scene.means), t(scene.log_scales), t(scene.quaternions), t(scene.opacity_logits),
          t(scene.sh)]
    cam = gsb.Camera(scene.world_to_camera, scene.position, scene.fx, scene.fy, scene.cx,
                     scene.cy, scene.width, scene.height)
    color, alpha, radii = gsb.rasterize_gaussians(*ps, cam)
    rng = np.random.default_rng(1)
    gc = rng.normal(size=color.shape).astype(np.float32)
    ga = rng.normal(size=alpha.shape).astype(np.float32)
    ((color * torch.from_numpy(gc).cuda()).sum() + (alpha * torch.from_numpy(ga).cuda()).sum()
     ).backward()
    o = cpu.render(scene)
    og = cpu.backward(scene, o, gc, ga)
    for p, ref in zip(ps, (og["means"], og["scales"], og["rotations"],
                           og["opacities"].reshape(-1, 1), og["sh"])):
        a = p.grad.detach().cpu().double().numpy().ravel()
        b = np.asarray(ref, np.float64).ravel()
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-3
