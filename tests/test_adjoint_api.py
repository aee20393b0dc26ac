"""Argument checks of reconstruct_differentiable that run before any device work
(warp-psr reconstruction_adjoint.py:69-88)."""
import pytest
import torch

from warp_psr_b200 import reconstruct_differentiable


def test_requires_tracked_inputs():
    p = torch.zeros(4, 3, dtype=torch.float64)
    with pytest.raises(ValueError, match="requires_grad"):
        reconstruct_differentiable(p, p.clone())


def test_tensor_options_rejected():
    p = torch.zeros(4, 3, dtype=torch.float64, requires_grad=True)
    with pytest.raises(ValueError, match="constant scalar"):
        reconstruct_differentiable(p, p.detach().clone(), point_weight=torch.ones(1))


def test_inputs_must_be_tensors():
    with pytest.raises(TypeError):
        reconstruct_differentiable([[0.0, 0.0, 0.0]], [[0.0, 0.0, 1.0]])
