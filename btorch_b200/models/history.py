"""Rolling spike history (API and layout of btorch/models/history.py:28-358).

Memory ``history`` has shape (*batch, max_delay, *n_neuron).  Circular mode
keeps a cursor (slot cursor-1 is the most recent spike); cat mode keeps the
most recent spike at index 0.  ``get_flattened(D)`` interleaves neurons and
delays [n0_d0, n0_d1, ..., n1_d0, ...], the row order of
expand_conn_for_delays.  The fused engine reads and writes this state when a
run starts and ends; stepping module by module uses these tensor moves.
"""

from __future__ import annotations

import torch

from .base import MemoryModule, normalize_n_neuron


class SpikeHistory(MemoryModule):
    def __init__(self, n_neuron, max_delay_steps: int = 5, use_circular_buffer: bool = True):
        super().__init__()
        self.n_neuron, self.size = normalize_n_neuron(n_neuron)
        self.max_delay = int(max_delay_steps)
        self.use_circular_buffer = use_circular_buffer
        self.register_memory("history", torch.tensor(0.0, dtype=torch.float32), (self.max_delay, *self.n_neuron))
        if use_circular_buffer:
            self.register_buffer("_cursor", torch.tensor(0, dtype=torch.long), persistent=False)

    def init_state(self, batch_size=None, dtype=None, device=None, persistent=False, skip_mem_name=()):
        super().init_state(batch_size, dtype, device, persistent, skip_mem_name)
        if self.use_circular_buffer:
            self._cursor = torch.tensor(0, dtype=torch.long, device=device)

    def reset(self, batch_size=None, dtype=None, device=None, skip_mem_name=(), inplace: bool = False):
        super().reset(batch_size, dtype, device, skip_mem_name, inplace=inplace)
        if self.use_circular_buffer:
            if inplace:
                self._cursor.zero_()
            else:
                self._cursor = torch.tensor(0, dtype=torch.long, device=self._cursor.device)

    def _nb(self) -> int:
        return self.history.ndim - 1 - len(self.n_neuron)

    def _delay_first(self) -> torch.Tensor:
        h = self.history
        nb = self._nb()
        if nb <= 0:
            return h
        return h.movedim(nb, 0)

    def update(self, spike: torch.Tensor) -> "SpikeHistory":
        if getattr(self, "history", None) is None:
            raise RuntimeError("SpikeHistory buffer not initialized. Call init_state() before first update().")
        spike = spike.to(self.history.dtype)
        nb = self._nb()
        if self.use_circular_buffer:
            # index ops with a device-side index: no host sync, so the update
            # can be captured in a CUDA graph
            h = self._delay_first()
            h.index_copy_(0, self._cursor.view(1), spike.unsqueeze(0))
            self._cursor.copy_((self._cursor + 1) % self.max_delay)
        else:
            h = self._delay_first()
            new = torch.cat([spike.unsqueeze(0), h[:-1]], dim=0)
            self.history = new.movedim(0, nb) if nb > 0 else new
        return self

    def get_delay(self, delay_steps: int) -> torch.Tensor:
        if delay_steps >= self.max_delay:
            raise IndexError(f"delay_steps ({delay_steps}) >= max_delay ({self.max_delay}). "
                             "Increase max_delay_steps or use smaller delays.")
        h = self._delay_first()
        if self.use_circular_buffer:
            return h.index_select(0, ((self._cursor - 1 - delay_steps) % self.max_delay).view(1)).squeeze(0)
        return h[delay_steps]

    def get_recent(self, n_steps: int) -> list[torch.Tensor]:
        if n_steps > self.max_delay:
            raise IndexError(f"n_steps ({n_steps}) > max_delay ({self.max_delay})")
        return [self.get_delay(d) for d in range(n_steps)]

    def get_flattened(self, n_delays: int) -> torch.Tensor:
        if n_delays > self.max_delay:
            raise IndexError(f"n_delays ({n_delays}) > max_delay ({self.max_delay})")
        st = torch.stack([self.get_delay(d) for d in range(n_delays)], dim=0)  # (D, *batch, *n)
        st = st.reshape(n_delays, *st.shape[1: st.ndim - len(self.n_neuron)], self.size)
        return st.movedim(0, -1).reshape(*st.shape[1:-1], self.size * n_delays)

    # -- engine interface: the last `k` spikes as [k][batch][n], index d = d steps ago
    def recent_block(self, k: int) -> torch.Tensor:
        return torch.stack([self.get_delay(d).reshape(-1, self.size) for d in range(k)])

    def store_recent_block(self, block: torch.Tensor, advance: int) -> None:
        """Set the history to what the reference holds after `advance` more
        update() calls whose last max_delay spikes are `block` [max_delay][batch][n]
        (index d = d steps ago).  Circular mode advances the cursor by `advance`."""
        k = block.shape[0]
        assert k == self.max_delay
        nb = self._nb()
        new = block.reshape(k, *self.history.shape[:nb], *self.n_neuron).to(self.history.dtype)
        if self.use_circular_buffer:
            self._cursor.copy_((self._cursor + advance) % k)
            order = (self._cursor - 1 - torch.arange(k, device=self._cursor.device)) % k
            h = self._delay_first()
            h[order] = new
        else:
            self.history = new.movedim(0, nb).contiguous() if nb > 0 else new.clone()
