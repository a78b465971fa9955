"""Surrogate spike functions (API of btorch/models/surrogate/base.py:6-62 and
sigmoid.py:13-66).

The neuron kernels evaluate the forward (Heaviside ``u >= 0``, or the smooth
``sigmoid(k * alpha * u)`` when ``spiking=False``) and the surrogate
derivative ``damping * 4 * s * (1 - s)`` with ``s = sigmoid(k * alpha * u)``,
``k = 2 ln(sqrt(2) + 1)``, so inside the fused and per-module steps these
objects only carry the parameters.  Called directly -- by a user's own
neuron model, as in the reference -- they apply the same forward and
surrogate backward as torch elementwise ops, in the reference's operation
order (the backward uses the surrogate derivative for the smooth forward
too).
"""

from __future__ import annotations

import math

import torch

SIG_K = 2.0 * math.log(math.sqrt(2.0) + 1.0)


class _Surrogate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, fn: "SurrogateFunctionBase"):
        ctx.fn = fn
        ctx.save_for_backward(x)
        return (x >= 0).to(x) if fn.spiking else fn.primitive(x)

    @staticmethod
    def backward(ctx, grad_output: torch.Tensor):
        (x,) = ctx.saved_tensors
        return ctx.fn.derivative(x, grad_output, ctx.fn.damping_factor), None


class SurrogateFunctionBase(torch.nn.Module):
    def __init__(self, alpha: float = 1.0, damping_factor: float = 1.0, spiking: bool = True):
        super().__init__()
        self.alpha = alpha
        self.damping_factor = damping_factor
        self.spiking = spiking

    def primitive(self, x: torch.Tensor) -> torch.Tensor:
        raise NotImplementedError

    def derivative(self, x: torch.Tensor, grad_output: torch.Tensor, damping_factor: float = 1.0) -> torch.Tensor:
        raise NotImplementedError

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        return _Surrogate.apply(x, self)


class Sigmoid(SurrogateFunctionBase):
    """Logistic surrogate; alpha is the inverse half-width (HWHM = 1/alpha)
    and the surrogate gradient at the threshold is `damping_factor`."""

    def __init__(self, alpha: float = 2.0, damping_factor: float = 1.0, spiking: bool = True):
        super().__init__(alpha=alpha, damping_factor=damping_factor, spiking=spiking)

    @property
    def slope(self) -> float:
        """k * alpha as the reference computes it (double product, used as fp32)."""
        return SIG_K * self.alpha

    def primitive(self, x: torch.Tensor) -> torch.Tensor:
        return torch.sigmoid(self.slope * x)

    def derivative(self, x: torch.Tensor, grad_output: torch.Tensor, damping_factor: float = 1.0) -> torch.Tensor:
        s = torch.sigmoid(self.slope * x)
        return grad_output * (damping_factor * 4.0 * s * (1.0 - s))


def sigmoid(x: torch.Tensor, alpha: float = 2.0, damping_factor: float = 1.0, spiking: bool = True) -> torch.Tensor:
    return Sigmoid(alpha=alpha, damping_factor=damping_factor, spiking=spiking)(x)


__all__ = ["Sigmoid", "SurrogateFunctionBase", "SIG_K", "sigmoid"]
