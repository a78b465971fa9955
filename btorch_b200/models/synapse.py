"""Synapse modules (API of btorch/models/synapse.py).

BasePSC (34-135), ExponentialPSC (138-187), DelayedPSC (537-623) and the
delay path of HeterSynapsePSC (626-761).  One ExponentialPSC step is one
kernel launch that evaluates psc + coef*((-psc)/tau_syn) + W z with the
reference's rounding, where W z comes from ``self.linear`` (SparseConn runs
the event-driven sparse kernels).  Inside RecurrentNN the whole step is run by
the fused engine instead (btorch_b200/models/engine.py).
"""

from __future__ import annotations

from collections.abc import Sequence

import torch

from . import environ
from ._ops import exp_euler_coef, psc_step
from .base import MemoryModule, flatten_neuron, normalize_n_neuron, unflatten_neuron
from .history import SpikeHistory


class BasePSC(MemoryModule):
    def __init__(self, n_neuron: int | Sequence[int], linear: torch.nn.Module, step_mode="s", backend="b200"):
        super().__init__()
        self.n_neuron, self.size = normalize_n_neuron(n_neuron)
        self.step_mode = step_mode
        self.backend = "b200" if backend == "torch" else backend
        self.linear = linear
        self.register_memory("psc", 0.0, self.n_neuron)

    def _wz(self, z: torch.Tensor) -> torch.Tensor:
        z_flat, leading = flatten_neuron(z, self.n_neuron, self.size)
        return unflatten_neuron(self.linear(z_flat), leading, self.n_neuron)

    def conductance_charge(self):
        raise NotImplementedError

    def current_charge(self, v=None):
        if v is not None:
            raise NotImplementedError("Only current-based PSC is supported.")
        return self.psc

    def single_step_forward(self, z: torch.Tensor):
        raise NotImplementedError

    def multi_step_forward(self, z_seq: torch.Tensor, kernel_len: int = 64):
        return torch.stack([self.single_step_forward(z) for z in z_seq])


class ExponentialPSC(BasePSC):
    """d psc/dt = -psc / tau_syn, exponential-Euler, plus W z each step."""

    def __init__(self, n_neuron, tau_syn, linear, step_mode="s", backend="b200"):
        super().__init__(n_neuron, linear, step_mode=step_mode, backend=backend)
        self.register_buffer("tau_syn", torch.as_tensor(tau_syn), persistent=False)

    def coefficients(self, dt: float):
        """(coef, tau) device fp32 vectors for the kernels; coef is rounded on
        the host exactly as the reference computes expm1(dt*lin)/lin."""
        tau = self.tau_syn.detach().float().reshape(-1).contiguous()
        return exp_euler_coef(self.tau_syn, dt, owner=self, name="psc"), tau

    def conductance_charge(self):
        coef, tau = self.coefficients(environ.get("dt"))
        self.psc = psc_step(self.psc.reshape(-1, self.size), None, coef, tau).reshape(self.psc.shape)
        return self.psc

    def single_step_forward(self, z: torch.Tensor):
        if self.psc is None:
            raise RuntimeError("ExponentialPSC.psc is not initialised; call init_net_state() first.")
        coef, tau = self.coefficients(environ.get("dt"))
        wz = self._wz(z)
        shape = self.psc.shape
        wz = torch.broadcast_to(wz, shape).reshape(-1, self.size)
        self.psc = psc_step(self.psc.reshape(-1, self.size), wz, coef, tau).reshape(shape)
        return self.psc


class DelayedPSC(MemoryModule):
    """Uniform delay of `max_delay_steps` in front of any PSC (SpikeHistory of
    max_delay_steps + 1 slots; the PSC sees z_{t - max_delay_steps})."""

    def __init__(self, psc: BasePSC, max_delay_steps: int = 1, use_circular_buffer: bool = False):
        super().__init__()
        self.psc_module = psc
        self.max_delay_steps = int(max_delay_steps)
        self.use_circular_buffer = use_circular_buffer
        self.history = (SpikeHistory(psc.n_neuron, max_delay_steps=self.max_delay_steps + 1,
                                     use_circular_buffer=use_circular_buffer)
                        if self.max_delay_steps > 1 else None)

    @property
    def n_neuron(self):
        return self.psc_module.n_neuron

    @property
    def size(self):
        return self.psc_module.size

    @property
    def step_mode(self):
        return self.psc_module.step_mode if hasattr(self, "psc_module") else self._step_mode

    @step_mode.setter
    def step_mode(self, value):
        if hasattr(self, "psc_module"):
            self.psc_module.step_mode = value
        else:
            self._step_mode = value

    @property
    def psc(self):
        return self.psc_module.psc

    def single_step_forward(self, z):
        if self.history is not None:
            self.history.update(z)
            z = self.history.get_delay(self.max_delay_steps)
        return self.psc_module.single_step_forward(z)

    def multi_step_forward(self, z_seq, kernel_len: int = 64):
        return torch.stack([self.single_step_forward(z) for z in z_seq])


class HeterSynapsePSC(BasePSC):
    """Receptor-expanded PSC with per-synapse delays through a delay-expanded
    connection matrix (rows pre * max_delay_steps + bin).  The fused engine
    implements n_receptor == 1 with an ExponentialPSC base."""

    def __init__(self, n_neuron, n_receptor: int, receptor_type_index, linear, base_psc=ExponentialPSC,
                 max_delay_steps: int = 1, use_circular_buffer: bool = False, step_mode="s", backend="b200",
                 **kwargs):
        super().__init__(n_neuron, linear, step_mode=step_mode, backend=backend)
        self.max_delay_steps = int(max_delay_steps)
        self.use_circular_buffer = use_circular_buffer
        self.history = (SpikeHistory(self.size, max_delay_steps=self.max_delay_steps,
                                     use_circular_buffer=use_circular_buffer)
                        if self.max_delay_steps > 1 else None)
        self.base_psc = base_psc(n_neuron=self.size * n_receptor, linear=linear, step_mode=step_mode,
                                 backend=backend, **kwargs)
        self.n_receptor = int(n_receptor)
        self.receptor_type_index = receptor_type_index

    def init_state(self, batch_size=None, dtype=None, device=None, persistent=True, skip_mem_name=()):
        super().init_state(batch_size, dtype, device, persistent, skip_mem_name=skip_mem_name)
        if self.history is not None:
            self.history.init_state(batch_size, dtype, device, persistent)

    def reset(self, batch_size=None, dtype=None, device=None, skip_mem_name=(), inplace: bool = False):
        super().reset(batch_size, dtype, device, skip_mem_name=skip_mem_name, inplace=inplace)
        if self.history is not None:
            self.history.reset(batch_size, dtype, device, inplace=inplace)

    def single_step_forward(self, z):
        lead = z.shape[: z.ndim - len(self.n_neuron)]
        z_flat = z.reshape(*lead, self.size)
        if self.history is not None:
            self.history.update(z_flat)
            z_flat = self.history.get_flattened(self.max_delay_steps)
        psc = self.base_psc.single_step_forward(z_flat)
        self.psc = psc.reshape(*lead, *self.n_neuron, self.n_receptor).sum(-1)
        return self.psc


__all__ = ["BasePSC", "ExponentialPSC", "DelayedPSC", "HeterSynapsePSC", "SpikeHistory"]
