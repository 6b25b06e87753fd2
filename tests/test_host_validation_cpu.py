"""Host-side argument checks of the training-loss, pruning and densification
entry points: they refuse bad inputs before any device work, so they run on
the CPU (no GPU, no CUDA library call)."""
import importlib

import pytest
import torch

gsb = importlib.import_module("photara-studio_b200")


def test_losses_refuse_host_tensors_and_bad_shapes():
    x = torch.zeros((3, 16, 16))
    with pytest.raises(ValueError, match="CUDA"):
        gsb.fused_l1_ssim(x, x)
    with pytest.raises(ValueError, match="CUDA"):
        gsb.ssim_metric(x, x)
    with pytest.raises(ValueError, match="CUDA"):
        gsb.compute_training_loss(x, x)


def test_training_loss_options_and_modes():
    o = gsb.TrainingLossOptions()
    # photara's TrainingLossSettings / TrainingOptions defaults
    assert (o.photometric_weight, o.ssim_weight, o.match_alpha_weight) == (1.0, 0.2, 0.25)
    assert o.geometry_epsilon == 1e-3 and o.alpha_mode == "masked"
    assert gsb.loss._ALPHA_MODES == {"validity": -1, "masked": 0, "transparent": 1}


def test_densify_apply_refuses_bad_inputs():
    d = gsb.densify
    assert d.SPLIT_MODES == {"adc_covariance": 0, "dense_tangent": 1, "igs_random": 2,
                             "long_axis": 3}
    with pytest.raises(ValueError, match="CUDA bool/uint8"):
        d.select_rows(torch.ones(8, dtype=torch.bool))
    with pytest.raises(ValueError, match="int32"):
        d.gather_rows(torch.zeros(4, dtype=torch.int64), [])
    with pytest.raises(ValueError, match="CUDA"):
        d.gather_rows(torch.zeros(4, dtype=torch.int32), [torch.zeros((4, 3))])
