"""CUDA-graph capture and replay of a stateful multi-step loop
(API of btorch/models/cudagraph.py:101-242).

The fused engine captures its own chunk launches (engine.run with
``cudagraph=True``).  This runner serves the per-module path: it records one
call of ``fn`` -- every kernel of every step of a chunk -- and replays it.

What a replay cannot see is what it hard-wires: the addresses of its inputs,
of the state it starts from and of everything it writes.  So

* each captured signature (shapes, dtypes, devices of the tensor arguments
  and the values of the others) owns static copies of the arguments and of
  the initial state, and every call copies the caller's values into them;
* the modules' state is rebound to the replay's final-state tensors after
  each replay (the cells rebind state every step, so those tensors live in
  the graph's memory pool);
* outputs live in that pool too and are cloned out unless the caller copies
  them itself before the next replay;
* the warm-up runs execute, so each starts from a fresh copy of the entry
  state, and module buffers that the loop advances in place (a history
  cursor) are restored after them; the replays then advance those buffers
  exactly as an eager call would.

Inference only: a replay rewrites its static buffers in place, which would
invalidate any autograd graph recorded over them.
"""

from __future__ import annotations

from typing import Any

import torch

from .functional import named_hidden_states, set_hidden_states

__all__ = ["CudaGraphRunner", "clone_graph_outputs"]


def clone_graph_outputs(obj: Any) -> Any:
    """Copy replay results out of the graph's memory pool."""
    if torch.is_tensor(obj):
        return obj.clone()
    if isinstance(obj, dict):
        return {k: clone_graph_outputs(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return type(obj)(clone_graph_outputs(v) for v in obj)
    return obj


class _Captured:
    __slots__ = ("graph", "args", "state_in", "state_out", "outputs")

    def __init__(self, graph, args, state_in, state_out, outputs):
        self.graph = graph
        self.args = args
        self.state_in = state_in
        self.state_out = state_out
        self.outputs = outputs


def _signature(args, kwargs):
    def one(v):
        return ("t", tuple(v.shape), v.dtype, str(v.device)) if torch.is_tensor(v) else ("v", v)

    return tuple(one(a) for a in args), tuple(sorted((k, one(v)) for k, v in kwargs.items()))


class CudaGraphRunner:
    """``runner(module, fn, args, kwargs)`` replays ``fn(*args, **kwargs)``,
    capturing it on first use of a signature; ``module`` owns the state that
    ``fn`` advances.  ``warmup`` eager runs precede a capture."""

    def __init__(self, warmup: int = 3):
        self.warmup = warmup
        self.entries: dict[tuple, _Captured] = {}

    @staticmethod
    def check_supported(module, args):
        if not torch.cuda.is_available():
            raise RuntimeError("cudagraph=True requires CUDA to be available.")
        devices = {a.device for a in args if torch.is_tensor(a)}
        if any(d.type != "cuda" for d in devices):
            raise RuntimeError(f"cudagraph=True requires all inputs on a CUDA device, got {devices}.")
        if torch.is_grad_enabled() and (any(a.requires_grad for a in args if torch.is_tensor(a))
                                        or any(p.requires_grad for p in module.parameters())):
            raise RuntimeError(
                "cudagraph=True is inference-only: each call rewrites the runner's static buffers in place, "
                "which invalidates any autograd graph recorded over them. Run under torch.no_grad() / "
                "torch.inference_mode().")
        for attr, why in (("grad_checkpoint", "the capture path would silently ignore it"),
                          ("save_grad_history", "its hooks only fire in the backward pass")):
            if getattr(module, attr, False):
                raise RuntimeError(f"cudagraph=True is incompatible with {attr}=True ({why}).")

    def _capture(self, module, fn, args, kwargs):
        state0 = {k: (v.detach().clone() if torch.is_tensor(v) else v)
                  for k, v in named_hidden_states(module).items()}
        buffers0 = [(b, b.detach().clone()) for _, b in module.named_buffers()]

        def restore():
            # fresh copies: a memory updated in place (a circular history)
            # would otherwise carry the warm-up's writes into the next run
            set_hidden_states(module, {k: (v.clone() if torch.is_tensor(v) else v) for k, v in state0.items()})
            for b, v in buffers0:
                if not torch.equal(b, v):  # untouched buffers keep their version
                    b.copy_(v)

        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(self.warmup):
                restore()
                fn(*args, **kwargs)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        restore()

        static_args = tuple(a.detach().clone() if torch.is_tensor(a) else a for a in args)
        state_in = {k: v.clone() for k, v in state0.items() if torch.is_tensor(v)}
        set_hidden_states(module, state_in)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            outputs = fn(*static_args, **kwargs)
        state_out = named_hidden_states(module)
        restore()  # capture only records: hand the module back its real state
        return _Captured(graph, static_args, state_in, state_out, outputs)

    def __call__(self, module, fn, args, kwargs=None, clone_outputs: bool = True):
        kwargs = kwargs or {}
        self.check_supported(module, args)
        key = _signature(args, kwargs)
        entry = self.entries.get(key)
        if entry is None:
            entry = self._capture(module, fn, args, kwargs)
            self.entries[key] = entry
        for dst, src in zip(entry.args, args):
            if torch.is_tensor(dst):
                dst.copy_(src)
        current = named_hidden_states(module)
        for k, buf in entry.state_in.items():
            buf.copy_(current[k])
        entry.graph.replay()
        set_hidden_states(module, entry.state_out)
        return clone_graph_outputs(entry.outputs) if clone_outputs else entry.outputs

    def reset(self):
        """Drop captured graphs and their memory pools."""
        self.entries.clear()
