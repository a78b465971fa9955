"""The per-module time loop (RecurrentNNAbstract via make_rnn) on the CPU with
a plain-torch cell: every unroll / chunk_size / grad_checkpoint / cpu_offload
/ save_grad_history combination gives the outputs, gradients and per-step
gradient history of the one-step-at-a-time loop, and the loop matches
torch.nn.RNNCell (the reference's tests/models/rnn/test_rnn_ops.py:47-170 and
test_rnn_parity.py:16-96)."""

import itertools

import pytest
import torch
from torch import nn

from btorch_b200.models.base import MemoryModule
from btorch_b200.models.functional import reset_net_state
from btorch_b200.models.rnn import make_rnn


class TanhCell(MemoryModule):
    """h <- tanh(W_x x + W_h h + b), state `h`."""

    def __init__(self, input_size, hidden_size):
        super().__init__()
        self.W_x = nn.Parameter(torch.randn(hidden_size, input_size) * 0.5)
        self.W_h = nn.Parameter(torch.randn(hidden_size, hidden_size) * 0.5)
        self.b = nn.Parameter(torch.randn(hidden_size) * 0.1)
        self.register_memory("h", torch.zeros(1), hidden_size)

    def single_step_forward(self, x):
        self.h = torch.tanh(x @ self.W_x.t() + self.h @ self.W_h.t() + self.b)
        return self.h


def _configs():
    for unroll, chunk, ckpt, offload, hist in itertools.product([1, 4, False], [None, 4, 8], [True, False],
                                                               [True, False], [True, False]):
        if unroll is not False and chunk is not None and chunk % unroll:
            continue
        yield dict(unroll=unroll, chunk_size=chunk, grad_checkpoint=ckpt, cpu_offload=offload,
                   save_grad_history=hist)


def _run(rnn, x):
    reset_net_state(rnn, batch_size=x.shape[1])
    out, _ = rnn(x)
    out[-1].sum().backward()
    return out


@pytest.mark.parametrize("config", list(_configs()), ids=lambda c: "-".join(f"{k}={v}" for k, v in c.items()))
def test_every_chunking_matches_step_by_step(config):
    torch.manual_seed(42)
    T, B, n_in, n_h = 16, 2, 3, 4
    base = make_rnn(TanhCell, unroll=1, save_grad_history=True, grad_state_names=["h"])(n_in, n_h)
    kw = dict(config, grad_state_names=["h"] if config["save_grad_history"] else None)
    test = make_rnn(TanhCell, **kw)(n_in, n_h)
    test.load_state_dict(base.state_dict())
    x0 = torch.randn(T, B, n_in, requires_grad=True)
    x1 = x0.detach().clone().requires_grad_(True)
    out0, out1 = _run(base, x0), _run(test, x1)
    torch.testing.assert_close(out1, out0, atol=1e-6, rtol=0)
    torch.testing.assert_close(x1.grad, x0.grad, atol=1e-6, rtol=0)
    for p in ("W_x", "W_h", "b"):
        torch.testing.assert_close(getattr(test.rnn_cell, p).grad, getattr(base.rnn_cell, p).grad, atol=1e-6,
                                   rtol=0)
    if config["save_grad_history"]:
        h0, h1 = base.get_grad_history()["h"], test.get_grad_history()["h"]
        assert len(h1) == T and all(g is not None for g in h1)
        for t in range(T):
            torch.testing.assert_close(h1[t], h0[t], atol=1e-6, rtol=0)
    else:
        assert test.get_grad_history() == {}


def test_grad_history_is_the_total_gradient_of_each_state():
    """Slot t holds dL/dh_t through the output and through h_{t+1}; the last
    step's is the loss gradient itself; names not listed are not recorded."""
    torch.manual_seed(0)
    T, B = 5, 2
    rnn = make_rnn(TanhCell, unroll=1, save_grad_history=True, grad_state_names=["h"])(3, 4)
    x = torch.randn(T, B, 3)
    reset_net_state(rnn, batch_size=B)
    out, _ = rnn(x)
    out[-1].sum().backward()
    hist = rnn.get_grad_history()["h"]
    torch.testing.assert_close(hist[-1], torch.ones(B, 4))
    # dL/dh_{t} = (dL/dh_{t+1} * (1 - h_{t+1}^2)) @ W_h
    W_h = rnn.rnn_cell.W_h.detach()
    for t in range(T - 1):
        want = (hist[t + 1] * (1 - out[t + 1].detach() ** 2)) @ W_h
        torch.testing.assert_close(hist[t], want, atol=1e-6, rtol=1e-5)
    rnn.clear_grad_history()
    assert rnn.get_grad_history() == {}
    # named but not saved: one empty slot per step, reset every call
    quiet = make_rnn(TanhCell, grad_state_names=["h"])(3, 4)
    reset_net_state(quiet, batch_size=B)
    quiet(x)
    assert quiet.get_grad_history() == {"h": [None] * T}


@pytest.mark.parametrize("T", [1, 5, 8, 10])
@pytest.mark.parametrize("unroll", [1, 4, 8, False])
def test_matches_torch_rnn_cell(T, unroll):
    torch.manual_seed(42)
    B, n_in, n_h = 2, 3, 4
    rnn = make_rnn(TanhCell, unroll=unroll)(n_in, n_h)
    ref = nn.RNNCell(n_in, n_h)
    with torch.no_grad():
        ref.weight_ih.copy_(rnn.rnn_cell.W_x)
        ref.weight_hh.copy_(rnn.rnn_cell.W_h)
        ref.bias_ih.copy_(rnn.rnn_cell.b)
        ref.bias_hh.zero_()
    x = torch.randn(T, B, n_in, requires_grad=True)
    xr = x.detach().clone().requires_grad_(True)
    out = _run(rnn, x)
    h = torch.zeros(B, n_h)
    outs = []
    for t in range(T):
        h = ref(xr[t], h)
        outs.append(h)
    out_r = torch.stack(outs)
    out_r[-1].sum().backward()
    torch.testing.assert_close(out, out_r, atol=1e-6, rtol=0)
    torch.testing.assert_close(x.grad, xr.grad, atol=1e-6, rtol=0)
    torch.testing.assert_close(rnn.rnn_cell.W_h.grad, ref.weight_hh.grad, atol=1e-6, rtol=0)


def test_chunk_guard_and_remainders():
    rnn = make_rnn(TanhCell, unroll=4, chunk_size=6)(3, 4)
    reset_net_state(rnn, batch_size=2)
    with pytest.raises(ValueError, match="must be a multiple of unroll"):
        rnn(torch.randn(10, 2, 3))
    for T, unroll, chunk in ((3, 4, None), (8, 2, 10), (10, 4, 8), (11, 4, 8)):
        rnn = make_rnn(TanhCell, unroll=unroll, chunk_size=chunk)(3, 4)
        reset_net_state(rnn, batch_size=2)
        x = torch.randn(T, 2, 3, requires_grad=True)
        out, _ = rnn(x)
        assert out.shape == (T, 2, 4)
        out.sum().backward()
        assert x.grad is not None


def test_make_rnn_forms():
    cls = make_rnn(TanhCell)
    assert cls.__name__ == "RNN_TanhCell"
    inst = make_rnn(TanhCell(3, 4))
    deco = make_rnn()(TanhCell)
    for m in (cls(3, 4), inst, deco(3, 4)):
        reset_net_state(m, batch_size=2)
        assert m(torch.randn(4, 2, 3))[0].shape == (4, 2, 4)
    with pytest.raises(TypeError):
        make_rnn(3)


class GainCell(MemoryModule):
    """h <- tanh(W_x x + W_h h) * g, with g either per step or fixed."""

    def __init__(self, n_in, n_h):
        super().__init__()
        self.inner = TanhCell(n_in, n_h)
        self.register_memory("h", torch.zeros(1), n_h)

    def single_step_forward(self, x, g):
        self.h = self.inner.single_step_forward(x) * g
        return self.h


def _manual(cell, x, g, stepped, B):
    reset_net_state(cell, batch_size=B)
    return torch.stack([cell(x[t], g[t] if stepped else g).clone() for t in range(x.shape[0])])


@pytest.mark.parametrize("chunk", [None, 3])
def test_loop_args_step_time_indexed_inputs_only(chunk):
    """Arguments whose first axis has the first argument's length are stepped,
    the others are passed to every step unchanged (rnn.py:69-80), also across
    chunks, and loop_args= overrides the detection."""
    torch.manual_seed(3)
    rnn = make_rnn(GainCell, unroll=1, chunk_size=chunk)(3, 4)
    T, B = 7, 2
    x = torch.randn(T, B, 3)
    for g, stepped in ((torch.rand(T, B, 4) + 0.5, True), (torch.rand(B, 4) + 0.5, False)):
        reset_net_state(rnn, batch_size=B)
        out, _ = rnn(x, g)
        torch.testing.assert_close(out, _manual(rnn.rnn_cell, x, g, stepped, B), atol=1e-6, rtol=0)
    # with as many samples as steps a per-sample gain [B, 4] looks time-indexed:
    # detection steps it, loop_args=(0,) keeps it fixed
    B = T
    x = torch.randn(T, B, 3)
    g = torch.rand(B, 4) + 0.5
    for loop_args, stepped in ((None, True), ((0,), False)):
        reset_net_state(rnn, batch_size=B)
        out, _ = rnn(x, g, loop_args=loop_args)
        torch.testing.assert_close(out, _manual(rnn.rnn_cell, x, g, stepped, B), atol=1e-6, rtol=0)
