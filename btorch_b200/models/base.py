"""Stateful-module substrate with the reference's API and state layout.

Mirrors btorch/models/base.py: StepModule (17-52), ParamBufferMixin (75-457,
scalar-or-per-neuron parameters with compact state_dict entries),
MemoryModule (643-962: registered state tensors of shape (*batch, *sizes),
init_state / capture-safe reset(inplace=True)), and BaseNode (967-1124:
charge -> adaptation -> fire -> reset).  The state tensors are plain CUDA
buffers; the kernels read and write them in place.
"""

from __future__ import annotations

from collections.abc import Callable, Sequence
from dataclasses import dataclass
from numbers import Number
from typing import Any

import numpy as np
import torch

from .surrogate import Sigmoid


class StepModule:
    """step_mode dispatch: "s" runs single_step_forward, "m" multi_step_forward."""

    def supported_step_mode(self) -> tuple[str, ...]:
        return ("s", "m")

    @property
    def step_mode(self) -> str:
        return self._step_mode

    @step_mode.setter
    def step_mode(self, value: str):
        if value not in self.supported_step_mode():
            raise ValueError(f'step_mode can only be {self.supported_step_mode()}, but got "{value}"!')
        self._step_mode = value

    def single_step_forward(self, x, *args, **kwargs):
        raise NotImplementedError

    def multi_step_forward(self, x_seq, *args, **kwargs):
        raise NotImplementedError

    def forward(self, *args, **kwargs):
        if self.step_mode == "s":
            return self.single_step_forward(*args, **kwargs)
        if self.step_mode == "m":
            return self.multi_step_forward(*args, **kwargs)
        raise ValueError(self.step_mode)


def normalize_n_neuron(n_neuron: int | Sequence[int]) -> tuple[tuple[int, ...], int]:
    n = (n_neuron,) if isinstance(n_neuron, int) else tuple(int(v) for v in n_neuron)
    if len(n) == 0:
        raise ValueError("n_neuron must contain at least one dimension.")
    return n, int(np.prod(n))


def flatten_neuron(x: torch.Tensor, n_neuron: tuple[int, ...], size: int):
    if len(n_neuron) == 1:
        return x, x.shape[:-1]
    leading = x.shape[: -len(n_neuron)]
    return x.reshape(*leading, size), leading


def unflatten_neuron(x: torch.Tensor, leading_shape, n_neuron: tuple[int, ...]):
    if len(n_neuron) == 1:
        return x
    return x.reshape(*leading_shape, *n_neuron)


def _is_uniform(t: torch.Tensor, atol: float = 1e-6) -> bool:
    if t.numel() <= 1:
        return True
    if t.dtype.is_floating_point:
        return bool(torch.allclose(t, t.reshape(-1)[0], atol=atol))
    return bool((t == t.reshape(-1)[0]).all())


class ParamBufferMixin(torch.nn.Module):
    """def_param: a named value stored as a trainable Parameter or a buffer, in
    its compact (scalar) or full per-neuron form (btorch/models/base.py:75-457).

    Checkpoint shape policy, so that state dicts interchange with the
    reference's:
    * only neuron-sized values (sizes == n_neuron) are compacted: a uniform one
      is saved as a scalar; values with extra axes keep their full shape and a
      compact checkpoint value is broadcast back to it;
    * trainable_shape "full" keeps the full shape on load (broadcasting a
      compact value), "scalar" keeps a scalar -- a non-scalar checkpoint is an
      error for a trainable scalar and replaces a buffer's storage;
    * "auto" (and every buffer) becomes a scalar when the loaded value is
      uniform and takes the loaded shape otherwise."""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self._param_shape_mode: dict[str, str] = {}
        self._param_allow_compact: dict[str, bool] = {}

    def _resolve_is_trainable(self, name, trainable_param):
        if isinstance(trainable_param, bool):
            return trainable_param
        if isinstance(trainable_param, set):
            return name in trainable_param
        return name in getattr(self, "trainable_param", set())

    def def_param(self, name: str, val, *, sizes=None, trainable_param=None, trainable_shape: str = "auto",
                  normalize_to_sizes: bool = False, **kwargs):
        if sizes is None:
            sizes = tuple(getattr(self, "n_neuron"))
        sizes = tuple(int(s) for s in sizes)
        if trainable_shape not in ("auto", "scalar", "full"):
            raise ValueError(f"Invalid trainable_shape={trainable_shape!r}.")
        trainable = self._resolve_is_trainable(name, trainable_param)
        t = torch.as_tensor(val, **kwargs)
        if t.dtype == torch.float64 and kwargs.get("dtype") is None:
            t = t.to(torch.get_default_dtype())
        if len(sizes) > 1:
            # a flat full value, or one value per neuron without the last axis
            if t.ndim == 1 and t.numel() == int(np.prod(sizes)):
                t = t.reshape(sizes)
            elif t.ndim == len(sizes) - 1 and tuple(t.shape) == sizes[:-1]:
                t = t[..., None]
            elif t.ndim == 1 and t.numel() == int(np.prod(sizes[:-1])):
                t = t.reshape(sizes[:-1] + (1,))
        try:
            torch.broadcast_shapes(tuple(t.shape), sizes)
        except RuntimeError as e:
            raise ValueError(f"{name} shape {tuple(t.shape)} is not broadcastable to {sizes}.") from e
        if trainable and trainable_shape == "full" and tuple(t.shape) != sizes:
            t = torch.broadcast_to(t, sizes).clone()
        if trainable and trainable_shape == "scalar":
            if not _is_uniform(t):
                raise ValueError(f"{name} with trainable_shape='scalar' must be uniform.")
            t = t.reshape(-1)[:1].reshape(())
        if normalize_to_sizes and trainable_shape != "scalar" and tuple(t.shape) != sizes:
            t = torch.broadcast_to(t, sizes).clone()
        if hasattr(self, name):
            delattr(self, name)
        self._param_shape_mode[name] = trainable_shape if trainable else "auto"
        self._param_allow_compact[name] = sizes == tuple(getattr(self, "n_neuron", sizes))
        if trainable:
            self.register_parameter(name, torch.nn.Parameter(t))
        else:
            self.register_buffer(name, t, persistent=True)

    def _rebind(self, name: str, value: torch.Tensor):
        """Replace the storage of `name` (its shape changes), keeping its kind."""
        cur = getattr(self, name)
        value = value.detach().clone().to(device=cur.device, dtype=cur.dtype)
        if name in self._parameters:
            rg = self._parameters[name].requires_grad
            delattr(self, name)
            self.register_parameter(name, torch.nn.Parameter(value, requires_grad=rg))
        else:
            persistent = name not in self._non_persistent_buffers_set
            delattr(self, name)
            self.register_buffer(name, value, persistent=persistent)

    def _save_to_state_dict(self, destination, prefix, keep_vars):
        super()._save_to_state_dict(destination, prefix, keep_vars)
        for name, mode in self._param_shape_mode.items():
            key = prefix + name
            if mode == "full" or not self._param_allow_compact.get(name, True) or key not in destination:
                continue
            v = destination[key]
            if torch.is_tensor(v) and v.numel() > 1 and _is_uniform(v):
                destination[key] = v.reshape(-1)[:1].reshape(())

    def _load_from_state_dict(self, state_dict, prefix, local_metadata, strict, missing_keys, unexpected_keys,
                              error_msgs):
        for name, mode in self._param_shape_mode.items():
            key = prefix + name
            if key not in state_dict or not hasattr(self, name) or not torch.is_tensor(state_dict[key]):
                continue
            loaded = state_dict[key]
            cur_shape, new_shape = tuple(getattr(self, name).shape), tuple(loaded.shape)
            if mode == "full" or not self._param_allow_compact.get(name, True):
                if new_shape != cur_shape:
                    try:
                        state_dict[key] = torch.broadcast_to(loaded, cur_shape).clone()
                    except RuntimeError:
                        self._rebind(name, loaded)
                continue
            if loaded.numel() == 1 or (mode == "auto" and _is_uniform(loaded)):
                scalar = loaded.reshape(-1)[:1].reshape(())
                state_dict[key] = scalar
                if cur_shape != ():
                    self._rebind(name, scalar)
            elif mode == "scalar" and name in self._parameters:
                error_msgs.append(f"{key}: received non-scalar checkpoint tensor for trainable_shape='scalar' "
                                  "trainable parameter.")
            elif new_shape != cur_shape:
                self._rebind(name, loaded)
        super()._load_from_state_dict(state_dict, prefix, local_metadata, strict, missing_keys, unexpected_keys,
                                      error_msgs)


@dataclass
class ResetValue:
    """How a memory is (re)initialised (btorch/models/base.py:564-578)."""

    value: Any
    sizes: tuple[int, ...]
    dtype: torch.dtype | None = None
    persistent: bool | None = None
    has_batch: bool = False


def _memory_var(rv: ResetValue, batch_size, **fmt) -> torch.Tensor:
    sizes = tuple(rv.sizes)
    if batch_size is not None:
        bs = (batch_size,) if isinstance(batch_size, int) else tuple(batch_size)
        sizes = bs + sizes
    if rv.dtype is not None:
        fmt["dtype"] = rv.dtype
    if callable(rv.value):
        v = torch.as_tensor(rv.value(sizes, batch_size=batch_size)).to(**fmt)
    elif rv.value is None:
        return torch.empty(sizes, **fmt)
    else:
        v = torch.as_tensor(rv.value, **fmt).detach().clone()
    if tuple(v.shape) != sizes:
        v = torch.broadcast_to(v, sizes).clone()
    return v


class MemoryModule(StepModule, torch.nn.Module):
    """Base of all stateful modules: memories registered by name, stored as
    buffers of shape (*batch, *sizes) (btorch/models/base.py:643-962)."""

    def __init__(self):
        super().__init__()
        self._memories_rv: dict[str, ResetValue] = {}
        self._backend = "torch"
        self._step_mode = "s"

    @property
    def supported_backends(self):
        return ("torch", "b200")

    @property
    def backend(self) -> str:
        return self._backend

    @backend.setter
    def backend(self, value: str):
        if value not in self.supported_backends:
            raise NotImplementedError(f"{value} is not a supported backend of {self._get_name()}!")
        self._backend = value

    def multi_step_forward(self, x_seq, *args, **kwargs):
        return torch.stack([self.single_step_forward(x, *args, **kwargs) for x in x_seq])

    def register_memory(self, name: str, value, sizes, dtype=None, persistent=None):
        assert not hasattr(self, name), f"{name} has been set as a member variable!"
        sizes = (sizes,) if isinstance(sizes, int) else tuple(sizes)
        if isinstance(value, Number):
            value = np.asarray(value)
        elif isinstance(value, Sequence) and not isinstance(value, str):
            value = np.asarray(value)
        self._memories_rv[name] = ResetValue(value=value, sizes=sizes, dtype=dtype, persistent=persistent)
        self.register_buffer(name, None, persistent=False)

    def set_reset_value(self, name: str, value, *, strict: bool = True, **kw):
        old = self._memories_rv.get(name)
        if isinstance(value, ResetValue):
            self._memories_rv[name] = value
            return
        if isinstance(value, Number):
            value = np.asarray(value)
        sizes = kw.get("sizes", old.sizes if old else None)
        if sizes is None:
            raise ValueError(f"'sizes' is required when registering new memory_rv '{name}'")
        if strict and old is not None and "sizes" in kw and tuple(kw["sizes"]) != old.sizes:
            raise ValueError(f"Memory_rv '{name}' sizes mismatch")
        self._memories_rv[name] = ResetValue(value=value, sizes=tuple(sizes),
                                             dtype=kw.get("dtype", old.dtype if old else None),
                                             persistent=kw.get("persistent", old.persistent if old else None))

    @torch.no_grad()
    def init_state(self, batch_size=None, dtype=None, device=None, persistent=False, skip_mem_name=()):
        skip = set(skip_mem_name)
        for key, rv in self._memories_rv.items():
            if key in skip:
                continue
            v = _memory_var(rv, batch_size, dtype=rv.dtype or dtype, device=device)
            self.register_buffer(key, v, persistent=bool(rv.persistent or persistent))

    def _batch_dims(self, key):
        buf = self._buffers.get(key)
        sizes = self._memories_rv[key].sizes
        if buf is None or tuple(buf.shape) == tuple(sizes):
            return None
        return tuple(buf.shape[: buf.ndim - len(sizes)])

    @torch.no_grad()
    def reset(self, batch_size=None, dtype=None, device=None, skip_mem_name=(), inplace: bool = False):
        """Reset every memory to its registered value.  inplace=True writes into
        the existing buffers (address-stable, capture-safe, no host copy for
        zero-valued memories) and cannot change their shape."""
        skip = set(skip_mem_name)
        for key, rv in self._memories_rv.items():
            if key in skip:
                continue
            buf = self._buffers.get(key)
            bs = batch_size if batch_size is not None else self._batch_dims(key)
            fmt = {"device": device or (buf.device if buf is not None else None),
                   "dtype": rv.dtype or dtype or (buf.dtype if buf is not None else None)}
            if not inplace or buf is None:
                setattr(self, key, _memory_var(rv, bs, **fmt))
                continue
            is_zero = rv.value is not None and not callable(rv.value) and not bool(torch.as_tensor(rv.value).any())
            if is_zero:
                target = ((bs,) if isinstance(bs, int) else tuple(bs or ())) + tuple(rv.sizes)
                if tuple(buf.shape) != target:
                    raise ValueError(f"reset(inplace=True) cannot resize memory '{key}' from {tuple(buf.shape)} "
                                     f"to {target}; call reset()/init_state() to (re)allocate.")
                buf.zero_()
            else:
                v = _memory_var(rv, bs, **fmt)
                if tuple(buf.shape) != tuple(v.shape):
                    raise ValueError(f"reset(inplace=True) cannot resize memory '{key}' from {tuple(buf.shape)} "
                                     f"to {tuple(v.shape)}; call reset()/init_state() to (re)allocate.")
                buf.copy_(v)

    @torch.no_grad()
    def reset_rows(self, rows) -> None:
        """Reset rows `rows` (ints) of the batch dimension of every memory to the
        registered value, in place; other rows are untouched.  Used to recycle
        one sample slot of a batched model for a new request.  Scalar reset
        values are written with fill_ (no host-to-device copy, so the call does
        not wait for work queued on the stream); array values are moved to the
        device once and cached."""
        cache = self.__dict__.setdefault("_bt_row_reset", {})
        for key, rv in self._memories_rv.items():
            buf = self._buffers.get(key)
            if buf is None:
                continue
            bd = self._batch_dims(key)
            if bd is None:
                continue
            if len(bd) != 1:
                raise ValueError(f"reset_rows needs one batch dimension, memory '{key}' has {bd}")
            scalar = rv.value is not None and not callable(rv.value) and np.asarray(rv.value).size == 1
            val = None
            if not scalar:
                val = cache.get(key)
                if val is None or val.device != buf.device or val.dtype != buf.dtype:
                    val = _memory_var(rv, None, dtype=buf.dtype, device=buf.device)
                    cache[key] = val
            for r in rows:
                row = buf.select(0, int(r))
                if scalar:
                    row.fill_(float(np.asarray(rv.value).reshape(())))
                else:
                    row.copy_(val)

    def memories(self):
        for name in self._memories_rv:
            yield self._buffers[name]

    def named_memories(self):
        for name in self._memories_rv:
            yield name, self._buffers[name]

    def detach(self):
        for key in self._memories_rv:
            if self._buffers.get(key) is not None:
                self._buffers[key] = self._buffers[key].detach()

    @property
    def _memories(self):
        return {name: self._buffers[name] for name in self._memories_rv}

    @_memories.setter
    def _memories(self, value: dict):
        for k, v in value.items():
            assert k in self._memories_rv
            setattr(self, k, v)

    @property
    def memories_rv(self):
        return self._memories_rv

    def set_memories_rv(self, value: dict, strict: bool = False):
        for k, v in value.items():
            assert k in self._memories_rv
            self.set_reset_value(k, v, strict=strict)

    def extra_repr(self):
        return ", ".join(f"{k}={rv.sizes}" for k, rv in self._memories_rv.items())


class BaseNode(ParamBufferMixin, MemoryModule):
    """Spiking neuron base: memory `v` (initialised to v_reset), parameters
    v_threshold / v_reset, surrogate, reset mode (btorch/models/base.py:967-1124)."""

    def __init__(self, n_neuron, v_threshold=1.0, v_reset=0.0, trainable_param=set(),
                 surrogate_function: Callable = Sigmoid(), detach_reset=False, hard_reset=False,
                 pre_spike_v=False, step_mode="s", backend="b200", device=None, dtype=None):
        super().__init__()
        self.n_neuron, self.size = normalize_n_neuron(n_neuron)
        self.register_memory("v", v_reset, self.n_neuron)
        self.pre_spike_v = pre_spike_v
        if pre_spike_v:
            self.register_memory("v_pre_spike", v_reset, self.n_neuron, persistent=False)
        self.trainable_param = set(trainable_param)
        fk = {"device": device, "dtype": dtype}
        self.def_param("v_threshold", v_threshold, sizes=self.n_neuron, trainable_param=self.trainable_param, **fk)
        self.def_param("v_reset", v_reset, sizes=self.n_neuron, trainable_param=self.trainable_param, **fk)
        self.detach_reset = detach_reset
        self.surrogate_function = surrogate_function
        self.hard_reset = hard_reset
        self.step_mode = step_mode
        self.backend = "b200" if backend == "torch" else backend

    def extra_repr(self):
        return (f"n_neuron={self.n_neuron}, step_mode={self.step_mode}, hard_reset={self.hard_reset}, "
                f"surrogate={self.surrogate_function.__class__.__name__}")

    def multi_step_forward(self, x_seq):
        return torch.stack([self.single_step_forward(x) for x in x_seq])
