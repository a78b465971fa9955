"""Surrogate spike functions (API of btorch/models/surrogate/base.py:28-62 and
sigmoid.py:32-56).

The neuron kernels evaluate the forward (Heaviside ``u >= 0``, or the smooth
``sigmoid(k * alpha * u)`` when ``spiking=False``) and the surrogate
derivative ``damping * 4 * s * (1 - s)`` with ``s = sigmoid(k * alpha * u)``,
``k = 2 ln(sqrt(2) + 1)``; these objects only carry the parameters.
"""

from __future__ import annotations

import math

import torch

SIG_K = 2.0 * math.log(math.sqrt(2.0) + 1.0)


class SurrogateFunctionBase(torch.nn.Module):
    def __init__(self, alpha: float = 1.0, damping_factor: float = 1.0, spiking: bool = True):
        super().__init__()
        self.alpha = alpha
        self.damping_factor = damping_factor
        self.spiking = spiking


class Sigmoid(SurrogateFunctionBase):
    """Logistic surrogate; alpha is the inverse half-width (HWHM = 1/alpha)."""

    def __init__(self, alpha: float = 2.0, damping_factor: float = 1.0, spiking: bool = True):
        super().__init__(alpha=alpha, damping_factor=damping_factor, spiking=spiking)

    @property
    def slope(self) -> float:
        """k * alpha as the reference computes it (double product, used as fp32)."""
        return SIG_K * self.alpha


__all__ = ["Sigmoid", "SurrogateFunctionBase", "SIG_K"]
