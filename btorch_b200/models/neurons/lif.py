"""LIF neuron (constructor and state of btorch/models/neurons/lif.py:29-200).

One step = one launch of the sm_100a neuron kernel: Euler charge
v + dt*((-(v - v_reset))/tau + x/c_m), Heaviside fire of
(v - v_th)/(v_th - v_reset) gated by (refractory == 0), hard or soft reset,
refractory = relu(refractory + s*tau_ref - dt) -- each op rounded as the
reference's eager CPU op.
"""

from __future__ import annotations

from collections.abc import Callable, Sequence

import torch

from .. import environ
from .._ops import neuron_step
from ..base import BaseNode
from ..surrogate import Sigmoid


class LIF(BaseNode):
    def __init__(self, n_neuron: int | Sequence[int], v_threshold=1.0, v_reset=0.0, c_m=1.0, tau=20.0,
                 tau_ref=None, trainable_param: set[str] = set(), surrogate_function: Callable = Sigmoid(),
                 detach_reset: bool = False, hard_reset: bool = False, pre_spike_v: bool = False,
                 step_mode: str = "s", backend: str = "b200", device=None, dtype=None):
        super().__init__(n_neuron=n_neuron, v_threshold=v_threshold, v_reset=v_reset,
                         trainable_param=trainable_param, surrogate_function=surrogate_function,
                         detach_reset=detach_reset, hard_reset=hard_reset, pre_spike_v=pre_spike_v,
                         step_mode=step_mode, backend=backend, device=device, dtype=dtype)
        fk = {"device": device, "dtype": dtype}
        self.def_param("c_m", c_m, sizes=self.n_neuron, trainable_param=self.trainable_param, **fk)
        self.def_param("tau", tau, sizes=self.n_neuron, trainable_param=self.trainable_param, **fk)
        self._use_refractory = tau_ref is not None
        if self._use_refractory:
            self.def_param("tau_ref", tau_ref, sizes=self.n_neuron, trainable_param=self.trainable_param, **fk)
            self.register_memory("refractory", 0.0, self.n_neuron)
        else:
            self.tau_ref = None

    def _state2d(self, name):
        t = getattr(self, name)
        if t is None:
            raise RuntimeError(f"{type(self).__name__}.{name} is not initialised; call init_net_state() first.")
        return t.reshape(-1, self.size)

    def single_step_forward(self, x: torch.Tensor):
        dt = environ.get("dt")
        shape = self.v.shape if self.v is not None else None
        v2 = self._state2d("v")
        x2 = x.reshape(-1, self.size)
        if x2.shape[0] != v2.shape[0]:
            x2 = torch.broadcast_to(x.reshape(-1, self.size), v2.shape)
        ref2 = self._state2d("refractory") if self._use_refractory else None
        gk2 = self._state2d("g_k") if hasattr(self, "g_k") and "g_k" in self._memories_rv else None
        if self.pre_spike_v:
            self.v_pre_spike = self.v.clone()
        spike, v_new, ref_new, gk_new = neuron_step(self, x2, v2, ref2, gk2, dt)
        self.v = v_new.reshape(shape)
        if ref_new is not None:
            self.refractory = ref_new.reshape(shape)
        if gk_new is not None:
            self.g_k = gk_new.reshape(shape)
        return spike.reshape(shape)
