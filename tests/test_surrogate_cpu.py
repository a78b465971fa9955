"""The Sigmoid surrogate called directly (a user's own neuron model does
this; the built-in neurons evaluate it inside their kernels): forward and
surrogate backward bit for bit against the reference's
(tests/golden/surrogate.npz), unit gradient at the threshold and
HWHM = 1/alpha (the reference's tests/models/test_surrogate.py:32-112)."""

import json

import numpy as np
import pytest
import torch

from btorch_b200.models import Sigmoid
from btorch_b200.models.surrogate import sigmoid
from tests import cases

G = cases.load("surrogate")
RUNS = json.loads(str(G["runs"]))


@pytest.mark.parametrize("i", range(len(RUNS)))
def test_matches_reference_bitwise(i):
    x = torch.tensor(G["x"], requires_grad=True)
    y = Sigmoid(**RUNS[i])(x)
    (y * torch.tensor(G["r"])).sum().backward()
    np.testing.assert_array_equal(y.detach().numpy(), G[f"y{i}"])
    np.testing.assert_array_equal(x.grad.numpy(), G[f"g{i}"])


@pytest.mark.parametrize("alpha", [0.5, 2.0, 7.0])
def test_unit_gradient_and_half_width(alpha):
    x = torch.tensor(0.0, requires_grad=True)
    Sigmoid(alpha=alpha)(x).backward()
    assert abs(x.grad.item() - 1.0) < 1e-6
    x = torch.linspace(0, 3.0 / alpha, 10000, requires_grad=True)
    sigmoid(x, alpha=alpha).sum().backward()
    hw = x.detach()[x.grad >= 0.5].max().item()
    assert abs(hw - 1.0 / alpha) < 0.02 / alpha


def test_damping_scales_the_gradient_only():
    x0 = torch.linspace(-2, 2, 9, requires_grad=True)
    x1 = x0.detach().clone().requires_grad_(True)
    y0, y1 = Sigmoid(damping_factor=1.0)(x0), Sigmoid(damping_factor=0.5)(x1)
    assert torch.equal(y0, y1) and torch.equal(y0, (x0 >= 0).float())
    y0.sum().backward()
    y1.sum().backward()
    torch.testing.assert_close(x1.grad, 0.5 * x0.grad)
