"""SpikeHistory (the module-level delay buffer whose semantics the engine's
device ring reproduces) on the CPU: circular and shift modes, delay lookup,
the neuron-major flattened layout that delay-expanded matrices index, batch
and neuron shapes, reset (the reference's tests/models/test_history.py)."""

import pytest
import torch

from btorch_b200.models.history import SpikeHistory

PUSHES = [[1.0, 0.0, 0.0], [0.0, 2.0, 0.0], [0.0, 0.0, 3.0], [4.0, 0.0, 0.0], [0.0, 5.0, 0.0]]


def _filled(circular, n=3, D=3, pushes=PUSHES):
    h = SpikeHistory(n_neuron=n, max_delay_steps=D, use_circular_buffer=circular)
    h.init_state(batch_size=1, dtype=torch.float32)
    for p in pushes:
        h.update(torch.tensor([p]))
    return h


def test_construction_and_buffer_layout():
    h = SpikeHistory(n_neuron=10, max_delay_steps=5)
    assert h.n_neuron == (10,) and h.size == 10 and h.max_delay == 5
    assert h.use_circular_buffer is True and hasattr(h, "_cursor")
    assert not hasattr(SpikeHistory(n_neuron=10, max_delay_steps=5, use_circular_buffer=False), "_cursor")
    h.init_state(batch_size=2, dtype=torch.float32)
    assert h.history.shape == (2, 5, 10) and h.history.dtype == torch.float32


def test_update_needs_init_state():
    h = SpikeHistory(n_neuron=10, max_delay_steps=5)
    s = torch.randn(2, 10)
    with pytest.raises(RuntimeError, match="not initialized"):
        h.update(s)
    h.init_state(batch_size=2, dtype=torch.float32)
    assert h.update(s) is h
    assert torch.equal(h.history[:, 0, :], s)


@pytest.mark.parametrize("circular", [True, False])
def test_delay_lookup_after_wraparound(circular):
    h = _filled(circular)
    for d in range(3):
        assert torch.equal(h.get_delay(d), torch.tensor([PUSHES[4 - d]]))
    if not circular:  # shift mode keeps the newest spike at index 0
        for d in range(3):
            assert torch.equal(h.history[:, d, :], torch.tensor([PUSHES[4 - d]]))
    with pytest.raises(IndexError, match="delay_steps .* >= max_delay"):
        h.get_delay(3)
    with pytest.raises(IndexError, match="n_delays .* > max_delay"):
        h.get_flattened(4)
    with pytest.raises(IndexError, match="n_steps .* > max_delay"):
        h.get_recent(4)


@pytest.mark.parametrize("circular", [True, False])
def test_flattened_is_neuron_major(circular):
    h = _filled(circular, n=2, D=3, pushes=[[1.0, 10.0], [2.0, 20.0], [3.0, 30.0]])
    # column n * D + d holds neuron n's spike of d steps ago
    assert torch.equal(h.get_flattened(3), torch.tensor([[3.0, 2.0, 1.0, 30.0, 20.0, 10.0]]))
    assert torch.equal(h.get_flattened(2), torch.tensor([[3.0, 2.0, 30.0, 20.0]]))


def test_batch_and_neuron_shapes():
    h = SpikeHistory(n_neuron=2, max_delay_steps=3)
    h.init_state(batch_size=(2, 3), dtype=torch.float32)
    h.update(torch.randn(2, 3, 2))
    assert h.get_flattened(3).shape == (2, 3, 6)

    h = SpikeHistory(n_neuron=3, max_delay_steps=3)
    h.init_state(dtype=torch.float32)
    s = torch.tensor([1.0, 2.0, 3.0])
    h.update(s).update(s * 2)
    assert h.history.shape == (3, 3) and torch.equal(h.get_delay(1), s)

    h = SpikeHistory(n_neuron=(4, 5), max_delay_steps=3)
    assert h.size == 20
    h.init_state(batch_size=2, dtype=torch.float64)
    assert h.history.shape == (2, 3, 4, 5) and h.history.dtype == torch.float64
    s = torch.randn(2, 4, 5, dtype=torch.float64)
    h.update(s)
    assert torch.equal(h.get_delay(0), s)
    h.update(torch.randn(2, 4, 5, dtype=torch.float64)).update(torch.randn(2, 4, 5, dtype=torch.float64))
    assert h.get_flattened(3).shape == (2, 60)


def test_reset_clears_buffer_and_cursor():
    h = _filled(True)
    h.reset()
    assert torch.all(h.history == 0) and h._cursor.item() == 0
