"""Constraint hooks (API of btorch/models/constrain.py:5-20)."""

import torch
from torch import nn


class HasConstraint:
    """Modules that project their parameters back onto a constraint set."""

    def constrain(self, *args, **kwargs):
        raise NotImplementedError()


def constrain_net(mod: nn.Module) -> None:
    """Apply every HasConstraint module's constraint (under no_grad)."""
    with torch.no_grad():
        for m in mod.modules():
            if isinstance(m, HasConstraint):
                m.constrain()
