"""ADC-IGS selection (photara-studio_b200/igs.py, igs_plan) on CPU tensors
against the NumPy restatement oracle/densify_igs_ref.py of the reference's
refinement (densification_igs.cpp:287-500, cuda_ops.cu:263-302).

The deterministic parts (prune and recycle masks, rescue, cap, candidates,
priority median, edge factors, the three weight vectors, the growth count)
must agree exactly; the weighted draws are checked by their invariants and,
for the Gumbel top-k, by their frequencies."""
import importlib

import numpy as np
import pytest
import torch

from oracle.densify_igs_ref import igs_reference

igs = importlib.import_module("photara-studio_b200.igs")
gsb = importlib.import_module("photara-studio_b200")


def _scene(n=4000, seed=0):
    rng = np.random.default_rng(seed)
    means = rng.uniform(-2, 2, (n, 3)).astype(np.float32)
    log_scales = rng.normal(-3.5, 0.5, (n, 3)).astype(np.float32)
    quats = rng.normal(size=(n, 4)).astype(np.float32)
    logits = rng.normal(-1.0, 2.5, (n, 1)).astype(np.float32)   # many below 1/255
    sh = rng.normal(0, 0.1, (n, 16, 3)).astype(np.float32)
    means[5] = [1e6, 0, 0]            # outside 100 x extent
    log_scales[6] = [8.0, -3, -3]     # larger than 100 x extent
    logits[7] = np.nan                # non-finite
    sh[8, 3, 1] = np.inf
    count = rng.integers(0, 4, n).astype(np.float32)
    gradient = (rng.exponential(0.002, n) * (count > 0)).astype(np.float32)
    screen = (rng.exponential(0.08, n) * (count > 0)).astype(np.float32)
    with np.errstate(divide="ignore"):
        priority = (np.maximum(np.log2(screen / 0.25), 0) * count).astype(np.float32)
    return dict(means=means, log_scales=log_scales, quats=quats, logits=logits, sh=sh,
                count=count, gradient=gradient, screen=screen, priority=priority)


def _plan(sc, iteration=1000, cap=3_000_000, seed=1, recycle=0.01):
    t = torch.from_numpy
    model = gsb.GaussianModel(t(sc["means"]), t(sc["log_scales"]), t(sc["quats"]),
                              t(sc["logits"]), t(sc["sh"]), 3)
    n = sc["means"].shape[0]
    stats = igs.IgsStats(n, "cpu")
    stats.t["count"] = t(sc["count"])
    stats.t["gradient"] = t(sc["gradient"])
    stats.t["max_screen_radius"] = t(sc["screen"])
    stats.t["priority"] = t(sc["priority"])
    opts = igs.IgsOptions(cap=cap, dense_recycle_fraction=recycle)
    g = torch.Generator().manual_seed(seed)
    plan = igs.igs_plan(model, stats, iteration, opts, extent=5.0, center=(0, 0, 0), gen=g)
    ref = igs_reference(sc["means"], sc["log_scales"], sc["quats"], sc["logits"], sc["sh"],
                        sc["count"], sc["gradient"], sc["priority"], sc["screen"], iteration,
                        5.0, (0, 0, 0), cap=cap, recycle_fraction=recycle)
    return plan, ref


@pytest.mark.parametrize("seed,recycle", [(0, 0.01), (1, 0.2), (2, 0.0)])
def test_masks_weights_and_counts_match_the_restatement(seed, recycle):
    sc = _scene(seed=seed)
    plan, ref = _plan(sc, seed=seed, recycle=recycle)
    assert np.array_equal(plan.keep.numpy(), ref["keep"])
    assert plan.pruned == ref["pruned"] and plan.capacity == ref["capacity"]
    for k in ("candidate", "oversized", "growth_mask"):
        assert np.array_equal(getattr(plan, k).numpy(), ref[k]), k
    assert plan.counts["median"] == pytest.approx(ref["median"], rel=1e-6)
    for k in ("edge", "replacement_weights", "growth_weights", "oversize_scores"):
        np.testing.assert_allclose(getattr(plan, k).numpy(), ref[k], rtol=1e-6, atol=0, err_msg=k)
    assert plan.desired_growth == ref["desired_growth"]
    # the rows the rule may never prune: a non-hard row of the highest opacity
    op = 1 / (1 + np.exp(-sc["logits"].reshape(-1).astype(np.float64)))
    best = int(np.nanargmax(op))
    assert plan.keep[best]
    for bad in (5, 6, 7, 8):
        assert not plan.keep[bad]


def test_parent_selection_invariants():
    sc = _scene(seed=3)
    plan, ref = _plan(sc, seed=3, recycle=0.05)
    parents = plan.parents.numpy()
    assert np.all(np.diff(parents) > 0)                      # unique, increasing
    assert len(parents) <= plan.capacity
    rw = ref["replacement_weights"]
    n_rep = plan.counts["replacement"]
    assert n_rep == min(plan.pruned, plan.capacity, int((rw > 0).sum()))
    # oversized parents: the top-ranked eligible scores after the replacements
    over = ref["oversize_scores"]
    chosen_over = set(parents[over[parents] > 0].tolist())
    assert plan.counts["oversized"] <= len(chosen_over)
    n_grow = plan.counts["growth"]
    assert n_grow <= ref["desired_growth"]
    gw = ref["growth_weights"]
    assert len(parents) == n_rep + plan.counts["oversized"] + n_grow
    # every parent is a candidate with a positive weight in some selection
    assert np.all((rw[parents] > 0) | (over[parents] > 0) | (gw[parents] > 0))


def test_cap_drops_least_opaque_and_capacity_zero_grows_nothing():
    sc = _scene(seed=4)
    n = sc["means"].shape[0]
    plan, ref = _plan(sc, cap=n // 2, seed=4)
    assert np.array_equal(plan.keep.numpy(), ref["keep"])
    assert int(plan.keep.sum()) == n // 2 and plan.capacity == 0
    assert plan.parents.numel() == 0


def test_growth_stops_after_the_growth_window():
    sc = _scene(seed=5)
    plan, ref = _plan(sc, iteration=15_000, seed=5)
    assert plan.growth_weights is None and "growth_weights" not in ref
    assert plan.counts["oversized"] == 0 and plan.counts["growth"] == 0


def test_gumbel_top_k_draws_in_proportion_to_weight():
    w = torch.tensor([0.0, 1.0, 2.0, 4.0, float("nan"), 8.0])
    g = torch.Generator().manual_seed(0)
    hits = np.zeros(6)
    trials = 20_000
    for _ in range(trials):
        hits[int(igs._gumbel_top(w, 1, g)[0])] += 1
    assert hits[0] == 0 and hits[4] == 0
    p = hits[[1, 2, 3, 5]] / trials
    np.testing.assert_allclose(p, np.array([1, 2, 4, 8]) / 15, atol=0.012)
    # k = 3 of the four eligible rows: never a repeated or ineligible row
    for _ in range(200):
        pick = igs._gumbel_top(w, 3, g).tolist()
        assert len(set(pick)) == 3 and not set(pick) & {0, 4}
