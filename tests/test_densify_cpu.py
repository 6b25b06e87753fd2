"""CPU tests of the densification oracle and host logic: the MLP adjoint
against central differences, the split's covariance preservation, the plain
ADC rule on hand-made cases, and the decision-log labelling. No GPU needed."""
import importlib

import numpy as np
import pytest
import torch

from oracle import densify_ref as D

trainer = importlib.import_module("photara-studio_b200.trainer")
densify = importlib.import_module("photara-studio_b200.densify")


def _weights(seed=0):
    rng = np.random.default_rng(seed)
    w = rng.normal(size=D.N_PARAMS) * 0.3
    return D.bf16_round(w).astype(np.float64)


def test_mlp_oracle_gradient_matches_central_differences():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(40, 8))
    y = rng.integers(0, 4, size=40)
    wr = rng.uniform(0.2, 2.0, size=40)
    w = _weights(2)
    _, g = D.mlp_loss_grad(x, y, wr, w, wr.sum())
    h = 1e-6
    idx = rng.choice(D.N_PARAMS, size=60, replace=False)
    idx = np.concatenate([idx, [D.OFF_B1, D.OFF_B2, D.OFF_B3, D.N_PARAMS - 1]])
    for p in idx:
        wp, wm = w.copy(), w.copy()
        wp[p] += h
        wm[p] -= h
        fd = (D.mlp_loss_grad(x, y, wr, wp, wr.sum())[0] -
              D.mlp_loss_grad(x, y, wr, wm, wr.sum())[0]) / (2 * h)
        assert abs(fd - g[p]) <= 1e-6 + 1e-5 * abs(g[p]), (p, fd, g[p])


def test_bf16_rounding_is_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], np.float32)
    got = D.bf16_round(vals)
    want = torch.from_numpy(vals).to(torch.bfloat16).float().numpy()
    assert np.array_equal(got, want)


def test_split_preserves_mixture_covariance_and_opacity():
    rng = np.random.default_rng(3)
    n = 6
    means = rng.normal(size=(n, 3))
    ls = rng.normal(-2, 0.5, size=(n, 3))
    q = rng.normal(size=(n, 4))
    logits = rng.normal(size=n)
    parents = [1, 4]
    m2 = np.concatenate([means, means[parents]])
    l2 = np.concatenate([ls, ls[parents]])
    q2 = np.concatenate([q, q[parents]])
    o2 = np.concatenate([logits, logits[parents]])
    M, Ls, O = D.split(m2, l2, q2, o2, parents, n)
    for c, p in enumerate(parents):
        c += n
        mix_mean = 0.5 * (M[p] + M[c])
        assert np.allclose(mix_mean, means[p])
        cov = 0.5 * (D.covariance(Ls[p], q[p]) + D.covariance(Ls[c], q[p]))
        off = M[c] - mix_mean
        cov += np.outer(off, off)
        assert np.allclose(cov, D.covariance(ls[p], q[p]), rtol=1e-9, atol=1e-12)
        a = D.sigmoid(logits[p])
        a1 = D.sigmoid(O[p])
        assert np.isclose(1 - (1 - a1) ** 2, 1 - (1 - a) ** np.sqrt(2), rtol=1e-9)
    untouched = [i for i in range(n) if i not in parents]
    assert np.array_equal(M[untouched], means[untouched])


def test_adc_rule_cases():
    ext = 2.0
    p = dict(grad_threshold=2e-4, percent_dense=0.01, extent=ext, prune_opacity=0.005,
             prune_world_scale=0.1, prune_screen=0.0, densify=1)
    ls = np.log(np.array([[0.001] * 3, [0.05] * 3, [0.001] * 3, [0.5] * 3, [0.001] * 3]))
    logits = np.array([0.0, 0.0, -8.0, 0.0, 0.0])
    stats = {"grad_acc": np.array([1e-3, 1e-3, 1e-3, 1e-3, 1e-5]),
             "count": np.array([2.0, 2, 2, 2, 2]), "max_screen": np.zeros(5)}
    act = D.adc_decide(ls, logits, stats, p)
    # clone (small), split (large), prune (opacity), prune (too big), keep (low grad)
    assert act.tolist() == [D.CLONE, D.SPLIT, D.PRUNE, D.PRUNE, D.KEEP]
    p["densify"] = 0
    assert D.adc_decide(ls, logits, stats, p).tolist() == [0, 0, 3, 3, 0]


def test_policy_fallback_rules():
    z = np.array([[5.0, 0, 0, 0], [0, 5.0, 0, 0], [0.1, 0.2, 0.0, 0.05], [0, 0, 5.0, 0],
                  [5.0, 0, 0, 0]])
    fallback = np.array([2, 0, 1, 0, 3])
    count = np.array([1.0, 1, 1, 0, 1])
    act = D.proposal_policy(z, fallback, count, 0.5)
    # confident keep; confident split; unconfident -> fallback; clone of unseen
    # -> fallback; hard prune always wins
    assert act.tolist() == [0, 1, 1, 0, 3]


def test_labels_from_logs_keeps_only_helpful_densifications():
    feats = torch.arange(6 * 8, dtype=torch.float32).reshape(6, 8)
    log = {"feats": feats,
           "action": torch.tensor([1, 2, 2, 3, 0, 0], dtype=torch.int32),
           "e_before": torch.tensor([1.0, 1.0, 1.0, 1.0, 1.0, 1.0]),
           "e_after": torch.tensor([0.5, 0.99, 0.2, 1.0, 1.0, 1.0]),
           "seen_after": torch.tensor([True, True, False, True, True, True])}
    F, Y, W = trainer.labels_from_logs([log], min_gain=0.05)
    rows = {int(f[0]) // 8: (int(y), float(w)) for f, y, w in zip(F, Y, W)}
    assert rows[0] == (densify.SPLIT, pytest.approx(0.5))
    assert rows[1][0] == densify.KEEP          # 1% gain: relabelled keep
    assert 2 not in rows                         # never seen after: no outcome
    assert rows[3][0] == densify.PRUNE and rows[4][0] == densify.KEEP


def test_time_to_psnr():
    h = [{"seconds": 1.0, "psnr": 20.0}, {"seconds": 2.0, "psnr": 25.0},
         {"seconds": 3.0, "psnr": 24.0}]
    assert trainer.time_to_psnr(h, 24.5) == 2.0
    assert trainer.time_to_psnr(h, 30.0) is None
