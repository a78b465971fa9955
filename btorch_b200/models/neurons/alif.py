"""ALIF neuron (constructor and state of btorch/models/neurons/alif.py:30-268).

One step = one launch: exponential-Euler charge with the conductance-based
adaptation term, g_k decay (exp-Euler with the host-rounded coefficient),
fire, reset, g_k += dg_k * s, refractory update.
"""

from __future__ import annotations

from collections.abc import Callable, Sequence

from ..surrogate import Sigmoid
from .lif import LIF


class ALIF(LIF):
    def __init__(self, n_neuron: int | Sequence[int], v_threshold=1.0, v_reset=0.0, c_m=1.0, g_leak=1.0,
                 E_leak=0.0, E_k=-70.0, g_k_init=0.0, tau_adapt=20.0, dg_k=0.0, tau_ref=None,
                 trainable_param: set[str] = set(), surrogate_function: Callable = Sigmoid(),
                 detach_reset: bool = False, hard_reset: bool = False, pre_spike_v: bool = False,
                 step_mode: str = "s", backend: str = "b200", device=None, dtype=None):
        super().__init__(n_neuron, v_threshold=v_threshold, v_reset=v_reset, c_m=c_m, tau=1.0, tau_ref=tau_ref,
                         trainable_param=trainable_param, surrogate_function=surrogate_function,
                         detach_reset=detach_reset, hard_reset=hard_reset, pre_spike_v=pre_spike_v,
                         step_mode=step_mode, backend=backend, device=device, dtype=dtype)
        del self.tau  # ALIF has no membrane tau parameter
        self._param_shape_mode.pop("tau", None)
        fk = {"device": device, "dtype": dtype}
        for name, val in (("g_leak", g_leak), ("E_leak", E_leak), ("E_k", E_k), ("tau_adapt", tau_adapt),
                          ("dg_k", dg_k)):
            self.def_param(name, val, trainable_param=self.trainable_param, **fk)
        self.register_memory("g_k", g_k_init, self.n_neuron)
