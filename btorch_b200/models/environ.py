"""Thread-local computation environment (API of btorch/models/environ.py:24-139).

``dt`` is read when a step is launched and baked into the kernels' fp32
coefficients."""

from __future__ import annotations

import functools
import threading
from typing import Any


class _State(threading.local):
    def __init__(self):
        self.settings: dict[str, Any] = {}
        self.contexts: dict[str, list] = {}


_STATE = _State()


class context:
    """Push key/values for the duration of a ``with`` block (or a decorated call)."""

    def __init__(self, **kwargs):
        self.kwargs = kwargs

    def __enter__(self):
        for k, v in self.kwargs.items():
            _STATE.contexts.setdefault(k, []).append(v)
        return all()

    def __exit__(self, exc_type, exc, tb):
        for k in self.kwargs:
            _STATE.contexts[k].pop()

    def __call__(self, func):
        @functools.wraps(func)
        def wrapped(*a, **kw):
            with self:
                return func(*a, **kw)

        return wrapped


def get(key: str, desc: str | None = None):
    stack = _STATE.contexts.get(key)
    if stack:
        return stack[-1]
    if key in _STATE.settings:
        return _STATE.settings[key]
    hint = (f"'{key}' is not found in the context. \nYou can set it by `environ.context({key}=value)` "
            f"locally or `environ.set({key}=value)` globally.")
    if desc is not None:
        hint += f" \nDescription: {desc}"
    raise KeyError(hint)


def all() -> dict:  # noqa: A001 -- reference name
    r = {k: v[-1] for k, v in _STATE.contexts.items() if v}
    for k, v in _STATE.settings.items():
        r.setdefault(k, v)
    return r


def set(**kwargs):  # noqa: A001 -- reference name
    _STATE.settings.update(kwargs)
