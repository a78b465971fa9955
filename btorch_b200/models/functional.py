"""Network-wide state helpers (API of btorch/models/functional.py:26-500)."""

from __future__ import annotations

import logging
from collections.abc import Sequence
from contextlib import contextmanager
from typing import Any

import torch
from torch import nn

from . import base


def _move_net(net: nn.Module, kwargs: dict) -> None:
    mv = {k: kwargs[k] for k in ("device", "dtype") if kwargs.get(k) is not None}
    if mv:
        net.to(**mv)


def init_net_state(net: nn.Module, batch_size: int | Sequence[int] | None = None, **kwargs):
    """init_state() on every MemoryModule in `net` (functional.py:26-61)."""
    _move_net(net, kwargs)
    for m in net.modules():
        if hasattr(m, "init_state") and callable(m.init_state):
            if not isinstance(m, base.MemoryModule):
                logging.warning(f"Trying to call `init_state()` of {m}, which is not base.MemoryModule")
            m.init_state(batch_size, **kwargs)


def reset_net(net: nn.Module, batch_size: int | Sequence[int] | None = None, **kwargs):
    """reset() on every MemoryModule (functional.py:64-98); inplace=True keeps
    buffer addresses (capture-safe)."""
    _move_net(net, kwargs)
    for m in net.modules():
        if hasattr(m, "reset") and callable(m.reset):
            m.reset(batch_size, **kwargs)


reset_net_state = reset_net


@contextmanager
def prepare_sparse_modules(net: nn.Module, batch_size: int | None = None):
    """Prepare sparse caches for one multi-step run (functional.py:104-124)."""
    from .linear import BaseSparseConn

    prepared = []
    try:
        for m in net.modules():
            if isinstance(m, BaseSparseConn):
                m.prepare_sparse(batch_size=batch_size)
                prepared.append(m)
        yield
    finally:
        for m in reversed(prepared):
            m.finish_sparse()


def _strip_self(names):
    return {s.removeprefix("self.").removeprefix("self") for s in names}


def named_hidden_states(mod: nn.Module, names: Sequence[str] | None = None, allow_buffer: bool = False,
                        clone: bool = False) -> dict[str, Any]:
    """Dotted dict of every memory (functional.py:224-250)."""
    names_set = _strip_self(set(names)) if names is not None else None
    ret = {}
    for name, m in mod.named_modules():
        if not (allow_buffer or isinstance(m, base.MemoryModule)):
            continue
        prefix = "" if name == "" else f"{name}."
        src = m._memories if isinstance(m, base.MemoryModule) else dict(m.named_buffers(recurse=False))
        for k, v in src.items():
            key = prefix + k
            if names_set is None or name in names_set or key in names_set:
                ret[key] = v.clone() if clone and torch.is_tensor(v) else v
    return ret


filter_hidden_states = named_memory_values = named_hidden_states


def set_hidden_states(mod: nn.Module, hidden_states: dict[str, Any], allow_buffer: bool = False,
                      inplace: bool = False):
    """Set memories from a dotted dict (functional.py:256-302)."""
    if hidden_states is None:
        return
    for name, value in hidden_states.items():
        if value is None:
            continue
        path = name.removeprefix("self.").removeprefix("self").split(".")
        m = mod
        for p in path[:-1]:
            m = getattr(m, p)
        leaf = path[-1]
        target = getattr(m, leaf, None) if leaf else m
        if isinstance(target, nn.Module) or leaf == "":
            target = m if leaf == "" else target
            for k, v in value.items():
                if inplace:
                    getattr(target, k).copy_(v)
                else:
                    setattr(target, k, v)
        elif inplace:
            getattr(m, leaf).copy_(value)
        else:
            setattr(m, leaf, value)


set_memory_values = set_hidden_states


def named_memory_reset_values(mod: nn.Module, names: Sequence[str] | None = None) -> dict[str, Any]:
    """Dotted dict of every memory's reset value (base.ResetValue), e.g. to
    save beside state_dict so a reloaded model resets to the same values
    (functional.py:311-326); `names` filters like named_hidden_states."""
    names_set = _strip_self(set(names)) if names is not None else None
    ret = {}
    for name, m in mod.named_modules():
        if not isinstance(m, base.MemoryModule):
            continue
        prefix = "" if name == "" else f"{name}."
        for k, rv in m.memories_rv.items():
            key = prefix + k
            if names_set is None or name in names_set or key in names_set:
                ret[key] = rv
    return ret


def set_memory_reset_values(mod: nn.Module, reset_values: dict[str, Any] | None, strict: bool = True):
    """Set reset values from a dotted dict (functional.py:329-351): "a.b.v"
    sets memory v of module a.b (a ResetValue, or a value keeping the
    registered sizes); a key naming a module ("" or "self" for `mod` itself)
    takes a dict of that module's memories.  `strict` is passed to
    set_reset_value."""
    if reset_values is None:
        return
    for name, value in reset_values.items():
        if value is None:
            continue
        path = name.removeprefix("self.").removeprefix("self")
        parent, _, leaf = path.rpartition(".")
        owner = mod.get_submodule(parent)
        if leaf == "" or leaf in owner._modules:
            target = owner if leaf == "" else owner._modules[leaf]
            assert isinstance(target, base.MemoryModule), f"{name or 'self'} is not a MemoryModule"
            target.set_memories_rv(value, strict=strict)
        else:
            assert isinstance(owner, base.MemoryModule), f"{parent or 'self'} is not a MemoryModule"
            owner.set_reset_value(leaf, value, strict=strict)


def detach_net(net: nn.Module):
    """Cut the autograd history of every memory (truncated BPTT boundary)."""
    for m in net.modules():
        if hasattr(m, "detach") and callable(m.detach) and isinstance(m, base.MemoryModule):
            m.detach()


__all__ = ["init_net_state", "reset_net", "reset_net_state", "prepare_sparse_modules", "named_hidden_states",
           "filter_hidden_states", "set_hidden_states", "named_memory_reset_values", "set_memory_reset_values",
           "detach_net", "reset_rows"]


@torch.no_grad()
def reset_rows(net: nn.Module, rows) -> None:
    """Reset batch rows `rows` of every memory in `net` to its registered
    value (MemoryModule.reset_rows): recycles sample slots of a batched model
    without touching the other samples' state."""
    rows = [int(r) for r in (rows.tolist() if torch.is_tensor(rows) else rows)]
    for m in net.modules():
        if isinstance(m, base.MemoryModule):
            m.reset_rows(rows)
