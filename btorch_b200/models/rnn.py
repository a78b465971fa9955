"""Recurrent time loop (API of btorch/models/rnn.py).

RecurrentNN.multi_step_forward runs the whole loop through the fused device
engine (btorch_b200/models/engine.py) when the model matches it and no
gradient is needed; otherwise it steps module by module -- each module's
step is one of the sm_100a kernels with a hand-written backward -- using the
reference's chunking: unroll blocks, large chunks with optional gradient
checkpointing per chunk (truncated-BPTT windows recompute their forward in
backward), optional CPU offload of per-chunk outputs and the per-step
gradient history of named states (rnn.py:85-106, 200-332).
"""

from __future__ import annotations

from collections.abc import Sequence

import torch
import torch.nn as nn
from torch.utils.checkpoint import checkpoint

from . import base, environ
from . import bptt as _bptt
from . import engine as _engine
from .cudagraph import CudaGraphRunner
from .functional import filter_hidden_states, named_hidden_states, prepare_sparse_modules, set_hidden_states


class RecurrentNNAbstract(base.MemoryModule):
    def __init__(self, update_state_names: Sequence[str] | None = None, step_mode="m", unroll: int | bool = 8,
                 chunk_size: int | None = None, cpu_offload: bool = False, grad_checkpoint: bool = False,
                 save_grad_history: bool = False, grad_state_names=None, cudagraph: bool = False,
                 cudagraph_warmup: int = 3, fused: bool = True):
        super().__init__()
        self.step_mode = step_mode
        self.update_state_names = update_state_names
        self.unroll = unroll
        self.chunk_size = chunk_size
        self.cpu_offload = cpu_offload
        self.grad_checkpoint = grad_checkpoint
        self.save_grad_history = save_grad_history
        self.grad_state_names = grad_state_names
        self._grad_history = {}
        self.cudagraph = cudagraph
        self.cudagraph_warmup = cudagraph_warmup
        self._cudagraph_runner = CudaGraphRunner(warmup=cudagraph_warmup)
        self.fused = fused
        # the persistent engine modes' status word (a bounded wait that gave
        # up): "sync" reads it at the end of every call (one host
        # synchronisation; the call raises), "deferred" copies it to the host
        # asynchronously and raises at a later call or at engine_status()
        self.engine_status_check = "sync"
        self._engine_pending_status = None
        self.last_engine_stats = None
        self.last_engine_direction = None
        self.last_path = None

    def single_step_forward(self, *args, **kwargs):
        raise NotImplementedError

    def _detect_loop_args(self, *args):
        if len(args) == 1:
            return args[0].shape[0], (0,)
        shapes = [a.shape[0] if torch.is_tensor(a) and a.ndim > 0 else None for a in args]
        T = shapes[0]
        assert T is not None
        return T, tuple(i for i, s in enumerate(shapes) if s == T)

    def _chunk_plan(self, *args, loop_args=None):
        if loop_args is None:
            T, loop_args = self._detect_loop_args(*args)
        else:
            T = args[loop_args[0]].shape[0]
        unroll = T if self.unroll is False else int(self.unroll)
        if self.chunk_size is None:
            large = unroll if self.grad_checkpoint else T
        else:
            large = self.chunk_size
            if self.unroll is not False and large % unroll != 0:
                raise ValueError(f"chunk_size ({large}) must be a multiple of unroll ({unroll})")
        return T, loop_args, unroll, large, (T + large - 1) // large

    def _start_grad_history(self, T: int):
        """A fresh gradient history per call (rnn.py:255-265): with
        grad_state_names, one slot per step for each named state (even
        without save_grad_history); otherwise empty until hooks add states."""
        if self.save_grad_history:
            self._grad_history = {}
        if self.grad_state_names:
            self._grad_history = {name: [None] * T for name in self.grad_state_names}

    def _hook_grad(self, name: str, tensor, t: int, T: int):
        """Record the gradient that reaches state `name` of step t -- through
        the returned stack and through the recurrence (rnn.py:97-106,
        319-326)."""
        if not self.save_grad_history or (self.grad_state_names is not None and name not in self.grad_state_names):
            return
        slots = self._grad_history.setdefault(name, [None] * T)
        if torch.is_tensor(tensor) and tensor.requires_grad:
            def hook(grad):
                if grad is not None:
                    slots[t] = grad.detach().clone()
                return grad

            tensor.register_hook(hook)

    def _process_chunk(self, *chunk_args, loop_args=(0,), grad_steps=None, **kwargs):
        """Step through one chunk.  grad_steps = (first step, T) registers the
        gradient-history hooks on each step's states."""
        T = chunk_args[loop_args[0]].shape[0]
        zs, states = [], {}
        a = list(chunk_args)
        for t in range(T):
            for i in loop_args:
                a[i] = chunk_args[i][t]
            z, st = self.single_step_forward(*a, **kwargs)
            zs.append(z)
            for k, v in st.items():
                states.setdefault(k, []).append(v)
                if grad_steps is not None:
                    self._hook_grad(k, v, grad_steps[0] + t, grad_steps[1])
        return zs, states

    def _checkpointed_chunk(self, *chunk_args, loop_args=(0,), grad_steps=None, **kwargs):
        """One chunk under activation checkpointing (rnn.py:177-197): the
        forward keeps only the chunk's inputs and entry state; backward
        recomputes the chunk from them.  The recomputation runs on the
        modules themselves, so it restores the modules' state afterwards --
        the reference leaves them at wherever the (possibly early-stopped)
        recomputation got to, which truncated BPTT would then continue from.
        Gradient-history hooks go on the first run's states: backward runs
        through that run's graph, the recomputation only refills it."""
        memories = named_hidden_states(self)
        env = environ.all()
        calls = [0]

        def _pure(env, memories, *inner):
            recompute = calls[0] > 0
            calls[0] += 1
            current = dict(named_hidden_states(self)) if recompute else None
            try:
                set_hidden_states(self, memories)
                with environ.context(**env):
                    zs, st = self._process_chunk(*inner, loop_args=loop_args,
                                                 grad_steps=None if recompute else grad_steps, **kwargs)
                return torch.stack(zs), {k: torch.stack(v) for k, v in st.items()}
            finally:
                if recompute:
                    set_hidden_states(self, current)

        return checkpoint(_pure, env, memories, *chunk_args, use_reentrant=False)

    def _modular_forward(self, *args, loop_args=None, **kwargs):
        T, loop_args, unroll, large, n_chunks = self._chunk_plan(*args, loop_args=loop_args)
        splits = {i: torch.split(args[i], large, dim=0) for i in loop_args}
        self._start_grad_history(T)
        all_z, all_st = [], {}
        for c in range(n_chunks):
            cargs = tuple(splits[i][c] if i in loop_args else args[i] for i in range(len(args)))
            grad_steps = (c * large, T) if self.save_grad_history else None
            if self.cudagraph:
                def fn(*inner):
                    zs, sts = self._process_chunk(*inner, loop_args=loop_args, **kwargs)
                    return torch.stack(zs), {k: torch.stack(v) for k, v in sts.items()}

                # offloading copies out of the graph pool itself
                z, st = self._cudagraph_runner(self, fn, cargs, clone_outputs=not self.cpu_offload)
            elif self.grad_checkpoint:
                z, st = self._checkpointed_chunk(*cargs, loop_args=loop_args, grad_steps=grad_steps, **kwargs)
            else:
                zs, sts = self._process_chunk(*cargs, loop_args=loop_args, grad_steps=grad_steps, **kwargs)
                z, st = torch.stack(zs), {k: torch.stack(v) for k, v in sts.items()}
            if self.cpu_offload:
                z = z.cpu()
                st = {k: v.cpu() for k, v in st.items()}
            all_z.append(z)
            for k, v in st.items():
                all_st.setdefault(k, []).append(v)
        cat = lambda xs: xs[0] if len(xs) == 1 else torch.cat(xs)  # noqa: E731
        self.last_path = "modular"
        return cat(all_z), {k: cat(v) for k, v in all_st.items()}

    def multi_step_forward(self, *args, loop_args=None, **kwargs):
        first = args[0]
        batch = first[0].numel() // first.shape[-1] if torch.is_tensor(first) and first.ndim >= 2 else None
        with prepare_sparse_modules(self, batch_size=batch):
            return self._modular_forward(*args, loop_args=loop_args, **kwargs)

    def get_grad_history(self):
        return self._grad_history

    def clear_grad_history(self):
        self._grad_history = {}


class RecurrentNN(RecurrentNNAbstract):
    """z = neuron(synapse.psc + inp(x)); synapse(z) every step (rnn.py:485-528)."""

    def __init__(self, neuron: nn.Module, synapse: nn.Module, syn_inp_module: nn.Module | None = None,
                 neuron_inp_module: nn.Module | None = None, *, update_state_names=None, unroll: int | bool = 8,
                 chunk_size: int | None = None, cpu_offload: bool = False, grad_checkpoint: bool = False,
                 allow_buffer=False, **kwargs):
        super().__init__(update_state_names=update_state_names, unroll=unroll, chunk_size=chunk_size,
                         cpu_offload=cpu_offload, grad_checkpoint=grad_checkpoint, **kwargs)
        self.neuron = neuron
        self.synapse = synapse
        self.neuron_inp_module = neuron_inp_module
        self.syn_inp_module = syn_inp_module
        self.allow_buffer = allow_buffer

    def single_step_forward(self, x, x_syn=None):
        if self.neuron_inp_module is not None:
            x = self.neuron_inp_module(x)
        if self.syn_inp_module is not None:
            x_syn = self.syn_inp_module(x_syn)
        z = self.neuron(self.synapse.psc + x)
        self.synapse(z if x_syn is None else z + x_syn)
        return z, filter_hidden_states(self, self.update_state_names, allow_buffer=self.allow_buffer)

    def engine_status(self):
        """Wait for the status of the last persistent-engine call checked in
        "deferred" mode and raise RuntimeError if a wait in it gave up."""
        _engine.check_pending_status(self, wait=True)

    def fused_plan(self):
        """The engine plan for this model, or (None, reason)."""
        return _engine.match(self)

    def multi_step_forward(self, *args, loop_args=None, sample_len=None, spikes_out: str = "dense",
                           engine_chunk: int | None = None, engine_stats: bool = False,
                           engine_profile: list | None = None, engine_chunk_hook=None, engine_choice=None,
                           **kwargs):
        """Run T = args[0].shape[0] steps.  Extensions over the reference:
        sample_len ([batch] steps per sample; later steps of a sample freeze its
        state and emit no spikes), spikes_out="bitmask" (return the spike raster
        as [T, batch, ceil(n/32)] int32 words), engine_stats (record per-step
        active counts in self.last_engine_stats), engine_choice (an
        autotune.EngineChoice to run instead of the tuner's)."""
        needs_grad = torch.is_grad_enabled() and (
            any(p.requires_grad for p in self.parameters())
            or any(torch.is_tensor(a) and a.requires_grad for a in args))
        extra = len(args) > 1 and any(a is not None for a in args[1:])
        if torch.is_tensor(args[0]) and args[0].ndim > 0:
            self._start_grad_history(int(args[0].shape[0]))
        plan, reason = (None, "disabled")
        if self.fused and not needs_grad and not extra and not kwargs and loop_args in (None, (0,)):
            plan, reason = _engine.match(self)
        if self.cudagraph and plan is None:
            # (the fused engine also takes host-resident input, streamed in chunks)
            CudaGraphRunner.check_supported(self, args)
        if plan is not None:
            self.last_path = "fused"
            return _engine.run(plan, self, args[0], sample_len=sample_len, chunk=engine_chunk,
                               spikes_out=spikes_out, stats=engine_stats, profile=engine_profile,
                               chunk_hook=engine_chunk_hook, choice=engine_choice)
        if sample_len is not None or spikes_out != "dense":
            raise NotImplementedError(f"sample_len / spikes_out need the fused engine ({reason})")
        self.last_fused_reason = reason
        if self.fused and needs_grad and not extra and not kwargs and loop_args in (None, (0,)):
            paths, why = _bptt.match(self)
            if paths is not None:
                out = _bptt.run(self, args[0], paths)
                if out is not None:
                    return out
            self.last_fused_reason = f"{reason}; fused BPTT: {why or 'buffers too large'}"
        return super().multi_step_forward(*args, loop_args=loop_args, **kwargs)


def make_rnn(obj=None, allow_buffer=False, **rnn_kwargs):
    """Wrap a single-step MemoryModule class/instance into a time loop (rnn.py:433-482)."""

    def _build(cell):
        class RNNWrapped(RecurrentNNAbstract):
            def __init__(self, *args, **kwargs):
                super().__init__(**rnn_kwargs)
                self.rnn_cell = cell(*args, **kwargs) if isinstance(cell, type) else cell

            def single_step_forward(self, *args, **kwargs):
                out = self.rnn_cell(*args, **kwargs)
                return out, filter_hidden_states(self.rnn_cell, self.update_state_names, allow_buffer=allow_buffer)

        RNNWrapped.__name__ = f"RNN_{getattr(cell, '__name__', type(cell).__name__)}"
        return RNNWrapped

    if isinstance(obj, type):
        return _build(obj)
    if isinstance(obj, nn.Module):
        return _build(obj)()
    if obj is None:
        return _build
    raise TypeError("`make_rnn` expects a module class, a module instance, or None as a decorator.")


__all__ = ["RecurrentNNAbstract", "RecurrentNN", "make_rnn"]
