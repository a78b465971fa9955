"""Synapse modules (API of btorch/models/synapse.py).

BasePSC (34-135), ExponentialPSC (138-187), DelayedPSC (537-623) and
HeterSynapsePSC (626-847).  One ExponentialPSC step is one
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
        if tau.numel() not in (1, self.size):
            # the kernels read one time constant per neuron (the reference's
            # broadcast against psc raises for other lengths)
            raise RuntimeError(f"ExponentialPSC tau_syn has {tau.numel()} values; expected 1 or {self.size}.")
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


def receptor_sum_ordered(psc: torch.Tensor) -> torch.Tensor:
    """Sum over the last axis (C values) in the order torch's CPU sum reduces a
    contiguous row of C floats, replayed with elementwise adds:
    C < 4 left to right; 4 <= C < 8 a_j = p_j (j < 4), p_4 .. added to a_0 in
    turn, then ((a_0 + a_1) + a_2) + a_3; C >= 8 a_j = p_j + p_{8+j} + ... over
    the whole groups of 8, the left-to-right sum of the tail added to a_0,
    then a_0 + ... + a_7 left to right (checked against torch.sum for C <= 39;
    the fused engine's receptor_sum is the same)."""
    C = psc.shape[-1]
    p = [psc[..., r] for r in range(C)]
    if C < 4:
        s = p[0]
        for q in p[1:]:
            s = s + q
        return s if C > 1 else s.clone()
    if C < 8:
        a0 = p[0]
        for q in p[4:]:
            a0 = a0 + q
        return ((a0 + p[1]) + p[2]) + p[3]
    full = C - C % 8
    a = list(p[:8])
    for r in range(8, full):
        a[r % 8] = a[r % 8] + p[r]
    if full < C:
        t = p[full]
        for q in p[full + 1:]:
            t = t + q
        a[0] = a[0] + t
    s = a[0]
    for q in a[1:]:
        s = s + q
    return s


def receptor_sum(psc: torch.Tensor) -> torch.Tensor:
    """HeterSynapsePSC's sum over the receptor axis with the rounding of the
    reference's psc.reshape(..., n, C).sum(-1) on the CPU
    (synapse.py:744-747): torch.sum itself on the CPU (and for C <= 2, where
    the order does not matter, or C >= 40), the same order replayed with
    elementwise adds on the GPU, whose sum kernels add in another order."""
    C = psc.shape[-1]
    if psc.device.type == "cpu" or C <= 2 or C >= 40:
        return psc.sum(-1)
    return receptor_sum_ordered(psc)


class HeterSynapsePSC(BasePSC):
    """Receptor-expanded PSC (synapse.py:626-847): base_psc runs on
    n * n_receptor columns (post * n_receptor + receptor, the layout of
    make_hetersynapse_conn) and psc is their receptor sum; with
    max_delay_steps > 1 the input goes through a spike history and a
    delay-expanded matrix (rows pre * max_delay_steps + bin).  The fused
    engine implements the ExponentialPSC base with up to 16 receptors."""

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

    def _flatten_input(self, z: torch.Tensor):
        """(flat input, leading shape, has receptor axis) for trailing shape
        n_neuron or (*n_neuron, n_receptor) (synapse.py:710-727)."""
        raw = tuple(self.n_neuron)
        expanded = (*raw, self.n_receptor)
        if tuple(z.shape[z.ndim - len(raw):]) == raw:
            lead = z.shape[: z.ndim - len(raw)]
            return z.reshape(*lead, self.size), lead, False
        if tuple(z.shape[z.ndim - len(expanded):]) == expanded:
            lead = z.shape[: z.ndim - len(expanded)]
            return z.reshape(*lead, self.size * self.n_receptor), lead, True
        raise RuntimeError("HeterSynapsePSC input shape mismatch. Expected trailing shape "
                           f"{raw} or {expanded}, got {tuple(z.shape)}.")

    def _validate_delayed_input(self, has_receptor_axis: bool, shape) -> None:
        if has_receptor_axis:
            raise RuntimeError("Delayed HeterSynapsePSC expects input without receptor axis. "
                               f"Expected trailing shape {tuple(self.n_neuron)}, got {tuple(shape)}.")

    def _reshape_sum_receptor(self, psc_flat: torch.Tensor, lead) -> torch.Tensor:
        return receptor_sum(psc_flat.reshape(*lead, *self.n_neuron, self.n_receptor))

    def single_step_forward(self, z):
        z_flat, lead, has_rec = self._flatten_input(z)
        if self.history is not None:
            self._validate_delayed_input(has_rec, z.shape)
            self.history.update(z_flat)
            z_flat = self.history.get_flattened(self.max_delay_steps)
        psc = self.base_psc.single_step_forward(z_flat)
        self.psc = self._reshape_sum_receptor(psc, lead)
        return self.psc

    def multi_step_forward(self, z_seq, kernel_len: int = 64):
        if self.history is not None:
            _, _, has_rec = self._flatten_input(z_seq)
            self._validate_delayed_input(has_rec, z_seq.shape)
            return torch.stack([self.single_step_forward(z) for z in z_seq])
        z_flat, lead, _ = self._flatten_input(z_seq)
        return self._reshape_sum_receptor(self.base_psc.multi_step_forward(z_flat, kernel_len=kernel_len), lead)

    def get_psc(self, receptor_type=None, psc: torch.Tensor | None = None, validate_nan: bool = True):
        """PSC of one receptor channel (synapse.py:763-830): None = the
        base PSC of every channel, an int = receptor index, a str = receptor
        type (connection mode), a (pre, post) tuple = receptor pair (neuron
        mode; the mode is read from receptor_type_index's columns)."""
        psc = psc if psc is not None else self.base_psc.psc
        if receptor_type is None:
            out = psc
        else:
            cols = self.receptor_type_index.columns
            neuron_mode = "pre_receptor_type" in cols and "post_receptor_type" in cols
            if isinstance(receptor_type, tuple):
                if not neuron_mode:
                    raise ValueError("Tuple receptor_type requires neuron mode (receptor_type_index must have "
                                     "'pre_receptor_type' and 'post_receptor_type' columns)")
                idx = self.receptor_type_index.set_index(["pre_receptor_type", "post_receptor_type"])
                r = idx.loc[tuple(receptor_type), "receptor_index"]
            elif isinstance(receptor_type, str):
                if neuron_mode:
                    raise ValueError("String receptor_type not supported in neuron mode. "
                                     "Use tuple (pre_receptor_type, post_receptor_type) instead.")
                r = self.receptor_type_index.set_index("receptor_type").loc[receptor_type, "receptor_index"]
            else:
                r = int(receptor_type)
            out = psc.view(*psc.shape[:-1], *self.n_neuron, self.n_receptor)[..., int(r)]
        if validate_nan and torch.isnan(out).any():
            raise ValueError("NaN values detected in PSC tensor")
        return out


__all__ = ["BasePSC", "ExponentialPSC", "DelayedPSC", "HeterSynapsePSC", "SpikeHistory", "receptor_sum"]
