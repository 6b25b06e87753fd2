"""Densification apply kernels on the library: the four split operators
(photara split_gaussians_kernel, cuda_ops.cu:1720-1845), the ADC decay
(cuda_ops.cu:1847-1861, 3388-3400) and the pruning row selection with the
optimizer state (select_training_rows_gpu, densification_adc_plus.cpp:68-77),
against the reference's own kernels (oracle/_ref, bit-identical: the same
per-Gaussian float32 expressions), the float64 restatement
(oracle/densify_apply_ref.py) and torch's nonzero / index_select."""
import numpy as np
import pytest
import torch

from helpers import gsb

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a GPU")]

ref = pytest.importorskip("oracle.reference")
D = pytest.importorskip("oracle.densify_apply_ref")
densify = gsb.densify


def _model(n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    r = lambda *s: torch.randn(s, device="cuda", generator=g)
    return dict(means=r(n, 3), log_scales=-3 + 0.7 * r(n, 3), opacity_logits=1.5 * r(n),
                quaternions=r(n, 4)), g


def _as_model(d):
    sh = torch.zeros((d["means"].shape[0], 16, 3), device="cuda")
    return gsb.GaussianModel(d["means"], d["log_scales"], d["quaternions"], d["opacity_logits"],
                             sh, 3)


@pytest.mark.skipif(not ref.loss_available(), reason="reference kernels not built")
@pytest.mark.parametrize("mode", ["adc_covariance", "dense_tangent", "igs_random", "long_axis"])
def test_split_matches_reference_kernel_and_float64(mode):
    n, m = 20000, 7000
    base, g = _model(n, 3 + len(mode))
    parents = torch.randperm(n, device="cuda", generator=g)[:m].to(torch.int32).contiguous()
    rs = torch.randn((m, 3), device="cuda", generator=g)
    screens = 40 * torch.rand((m,), device="cuda", generator=g)
    kw = dict(random_samples=rs, screen_sizes=screens if mode == "adc_covariance" else None,
              minimum_opacity=1e-6, split_at_screen_size=12.0 if mode == "adc_covariance" else 0,
              split_opacity_k=0.55)
    mk = lambda: ({k: v.clone() for k, v in base.items()},
                  {k: v[parents.long()].clone() for k, v in base.items()})
    p_ours, c_ours = mk()
    densify.split_gaussians(_as_model(p_ours), _as_model(c_ours), parents, mode, **kw)
    p_ref, c_ref = mk()
    ref.split_gaussians(p_ref, c_ref, parents, mode, **kw)
    torch.cuda.synchronize()
    for k in ("means", "log_scales", "opacity_logits"):
        assert torch.equal(p_ours[k], p_ref[k]), (mode, k)
        assert torch.equal(c_ours[k], c_ref[k]), (mode, k)
    npk = {k: (v.cpu().numpy() if torch.is_tensor(v) else v) for k, v in kw.items()}
    P, Cc = D.split({k: v.cpu().numpy() for k, v in base.items()},
                    {k: v[parents.long()].cpu().numpy() for k, v in base.items()},
                    parents.cpu().numpy(), mode, **npk)
    for k in ("means", "log_scales", "opacity_logits"):
        for got, exp in ((p_ours[k], P[k]), (c_ours[k], Cc[k])):
            err = np.abs(got.cpu().numpy().astype(np.float64) - exp)
            assert err.max() <= 2e-5 * (np.abs(exp).max() + 1.0), (mode, k, err.max())


@pytest.mark.skipif(not ref.loss_available(), reason="reference kernels not built")
def test_adc_decay_matches_reference_kernel_and_float64():
    base, _ = _model(100003, 9)
    a = {k: v.clone() for k, v in base.items()}
    b = {k: v.clone() for k, v in base.items()}
    densify.apply_adc_decay(_as_model(a), 0.013, 0.021)
    ref.adc_decay(b["log_scales"], b["opacity_logits"], 0.013, 0.021)
    torch.cuda.synchronize()
    assert torch.equal(a["log_scales"], b["log_scales"])
    assert torch.equal(a["opacity_logits"], b["opacity_logits"])
    ls, lo = D.adc_decay(base["log_scales"].cpu().numpy(), base["opacity_logits"].cpu().numpy(),
                         0.013, 0.021)
    assert np.abs(a["log_scales"].cpu().numpy() - ls).max() < 1e-5
    # compared as opacities: sigmoid(l) - decay cancels in float32 for
    # opacities near the decay, which the logit of the difference magnifies
    got = 1 / (1 + np.exp(-a["opacity_logits"].cpu().numpy().astype(np.float64)))
    assert np.abs(got - 1 / (1 + np.exp(-lo))).max() < 1e-6


@pytest.mark.parametrize("n", [0, 1, 1023, 1024, 1025, 70001, 3_000_017])
def test_select_and_gather_rows_match_torch(n):
    g = torch.Generator(device="cuda").manual_seed(n + 1)
    keep = torch.rand((n,), device="cuda", generator=g) > 0.37
    idx = densify.select_rows(keep)
    assert torch.equal(idx.long(), torch.nonzero(keep).flatten())
    arrays = [torch.randn((n, 3), device="cuda", generator=g),
              torch.randn((n,), device="cuda", generator=g),
              torch.randn((n, 16, 3), device="cuda", generator=g).half(),
              torch.randint(0, 255, (n, 16, 3), device="cuda", generator=g).to(torch.uint8),
              torch.randn((n, 4), device="cuda", generator=g)]
    out = densify.gather_rows(idx, arrays)
    for a, o in zip(arrays, out):
        assert torch.equal(o, a.index_select(0, idx.long()))
    # tail rows (new Adam moments) come back zero
    out = densify.gather_rows(idx, arrays[:2], rows=idx.numel() + 5)
    for a, o in zip(arrays[:2], out):
        assert torch.equal(o[:idx.numel()], a.index_select(0, idx.long()))
        assert not o[idx.numel():].any()


def test_select_training_rows_keeps_moments_with_rows():
    n = 50000
    base, g = _model(n, 21)
    model = _as_model(base)
    model.sh.normal_(generator=g)
    adam = densify.AdamState.zeros(model)
    for v in list(adam.structure.values()):
        v.normal_(generator=g)
    adam.sh["first"].copy_(torch.randn(adam.sh["first"].shape, device="cuda", generator=g))
    adam.sh["packed"].random_(0, 255, generator=g)
    adam.sh["bounds"].normal_(generator=g)
    keep = torch.rand((n,), device="cuda", generator=g) > 0.5
    m2, a2 = densify.select_training_rows(model, adam, keep)
    sel = torch.nonzero(keep).flatten()
    for f in ("means", "log_scales", "quaternions", "opacity_logits", "sh"):
        assert torch.equal(getattr(m2, f), getattr(model, f).index_select(0, sel))
    for k, v in adam.structure.items():
        assert torch.equal(a2.structure[k], v.index_select(0, sel))
    for k, v in adam.sh.items():
        assert torch.equal(a2.sh[k], v.index_select(0, sel))
