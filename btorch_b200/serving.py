"""Continuous-batching simulation server for recurrent spiking networks.

Requests name a network, carry a stimulus (input current or input-channel
activity, [steps, c_in]) and run for their own number of steps.  Every
network is a `NetworkPool`: one RecurrentNN whose batch dimension is a set of
request slots, its neuron, synapse and delay state resident in HBM
([slots, n] per state variable).  The server loop

* admits queued requests in arrival order as soon as their network has a free
  slot and their device bytes (stimulus + spike raster) fit in the HBM
  budget; admission recycles the slot's rows of every state tensor
  (functional.reset_rows), leaving the other requests' state untouched;
* advances each pool by one tick -- `chunk` steps of all its occupied slots
  in shared launches (the fused engine, a CUDA graph per pool when enabled),
  with per-slot step counts (sample_len) so that a request that ends inside
  the tick freezes there and an empty slot does nothing;
* runs every pool on its own CUDA stream, so the ticks of different networks
  overlap on the device, and keeps at most `max_inflight` ticks queued per
  pool so that new arrivals are admitted promptly;
* retires a request when the tick that completed it has finished on the
  device (CUDA event), frees its slot and budget and records its latency.

Per-sample computations are independent in the engine (state, history and
spike sets are per sample; the gather modes sum in a fixed order per neuron,
and scatter sums are exact on dyadic weights), so a request's raster is the
same alone and in any mix of concurrent requests.

The reference has no serving layer; this drives the reference's module API
(RecurrentNN over MemoryModule state, btorch/models/rnn.py:485-528,
btorch/models/base.py:643-962) as per-slot device state.
"""

from __future__ import annotations

import heapq
import time
from collections import deque
from dataclasses import dataclass, field

import torch

from .models import engine, environ
from .models.functional import init_net_state, named_hidden_states, reset_rows


@dataclass
class SimRequest:
    network: str
    stimulus: torch.Tensor          # [steps, c_in] float32, host or device
    arrival: float = 0.0            # seconds after the server starts
    rid: int = -1
    # filled by the server
    raster: torch.Tensor | None = None  # [steps, ceil(n / 32)] int32 spike bitmaps (device)
    t_admit: float | None = None
    t_done: float | None = None
    slot: int | None = None
    pos: int = 0                    # steps already issued

    @property
    def steps(self) -> int:
        return int(self.stimulus.shape[0])

    @property
    def latency(self) -> float | None:
        return None if self.t_done is None else self.t_done - self.arrival


class NetworkPool:
    """One network with `slots` request slots; see the module docstring."""

    def __init__(self, name: str, rnn, slots: int, chunk: int = 128, device="cuda", cudagraph: bool = True,
                 max_inflight: int = 2):
        self.name = name
        self.rnn = rnn
        self.slots = int(slots)
        plan, reason = rnn.fused_plan()
        if plan is None:
            raise ValueError(f"network {name!r} does not run on the fused engine: {reason}")
        # a tick is a whole number of captured chunks
        self.chunk = engine.graph_chunk(plan.n_bins, chunk) if cudagraph else int(chunk)
        self.device = torch.device(device)
        self.max_inflight = max_inflight
        rnn.cudagraph = cudagraph
        init_net_state(rnn, batch_size=self.slots, dtype=torch.float32, device=self.device)
        self.n = rnn.neuron.size
        inp = rnn.neuron_inp_module
        self.c_in = inp.in_features if inp is not None else self.n
        self.words = (self.n + 31) // 32
        self.stream = torch.cuda.Stream(self.device)
        self.x_tick = torch.zeros((self.chunk, self.slots, self.c_in), device=self.device)
        self.lens = torch.zeros(self.slots, dtype=torch.int64, device=self.device)
        # pinned staging for the per-tick step counts: a ring one longer than
        # the ticks in flight, so a buffer is reused only after its tick ended
        self._lens_host = [torch.zeros(self.slots, dtype=torch.int64).pin_memory()
                           for _ in range(max_inflight + 1)]
        self.free = list(range(self.slots))
        self.active: dict[int, SimRequest] = {}
        self.inflight: deque = deque()   # (event, [requests finished by that tick])
        self.ticks = 0
        self.events = 0                  # synaptic events, summed from engine stats at retirement
        self._stat_parts = []

    # -- accounting --------------------------------------------------------
    def state_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in named_hidden_states(self.rnn).values()
                   if torch.is_tensor(t))

    def request_bytes(self, req: SimRequest) -> int:
        """Device bytes a request holds while admitted: its stimulus and raster."""
        return req.steps * (self.c_in * 4 + self.words * 4)

    # -- slot lifecycle ------------------------------------------------------
    def admit(self, req: SimRequest, now: float) -> None:
        slot = self.free.pop(0)
        req.slot, req.t_admit, req.pos = slot, now, 0
        with torch.cuda.stream(self.stream):
            reset_rows(self.rnn, [slot])
            req.stimulus = req.stimulus.to(self.device, torch.float32, non_blocking=True)
            req.raster = torch.empty((req.steps, self.words), dtype=torch.int32, device=self.device)
        self.active[slot] = req

    def busy(self) -> bool:
        return bool(self.active) or bool(self.inflight)

    def can_tick(self) -> bool:
        return bool(self.active) and len(self.inflight) < self.max_inflight

    def tick(self) -> None:
        """Issue `chunk` steps of every occupied slot on this pool's stream."""
        K = self.chunk
        lens = [0] * self.slots
        finished = []
        with torch.cuda.stream(self.stream), torch.inference_mode(), environ.context(dt=1.0):
            for slot, req in self.active.items():
                kc = min(K, req.steps - req.pos)
                lens[slot] = kc
                self.x_tick[:kc, slot].copy_(req.stimulus[req.pos:req.pos + kc])
            staged = self._lens_host[self.ticks % len(self._lens_host)]
            staged.copy_(torch.tensor(lens, dtype=torch.int64))
            self.lens.copy_(staged, non_blocking=True)
            raster, _ = self.rnn(self.x_tick, sample_len=self.lens, spikes_out="bitmask", engine_stats=True)
            self._stat_parts.append(self.rnn.last_engine_stats[:, 1].sum())
            for slot, req in list(self.active.items()):
                kc = lens[slot]
                req.raster[req.pos:req.pos + kc].copy_(raster[:kc, slot])
                req.pos += kc
                if req.pos >= req.steps:
                    finished.append(req)
                    del self.active[slot]
            ev = torch.cuda.Event()
            ev.record(self.stream)
        self.inflight.append((ev, finished))
        self.ticks += 1

    def retire(self, now: float) -> list[SimRequest]:
        """Requests whose last tick has finished on the device."""
        done = []
        while self.inflight and self.inflight[0][0].query():
            _, finished = self.inflight.popleft()
            for req in finished:
                req.t_done = now
                self.free.append(req.slot)
                done.append(req)
        return done

    def drain_events(self) -> int:
        if self._stat_parts:
            self.events += int(torch.stack(self._stat_parts).sum())
            self._stat_parts = []
        return self.events


@dataclass
class ServeReport:
    requests: list = field(default_factory=list)
    wall_s: float = 0.0
    events: int = 0
    ticks: dict = field(default_factory=dict)

    def latency_ms(self, q: float) -> float:
        lat = sorted(r.latency for r in self.requests)
        if not lat:
            return float("nan")
        i = min(len(lat) - 1, max(0, int(round(q * (len(lat) - 1)))))
        return lat[i] * 1e3

    def summary(self) -> dict:
        return {"requests": len(self.requests), "wall_s": self.wall_s,
                "p50_ms": self.latency_ms(0.50), "p99_ms": self.latency_ms(0.99),
                "events_per_s": self.events / self.wall_s if self.wall_s > 0 else 0.0,
                "ticks": self.ticks}


class SimulationServer:
    """Admission by HBM budget + continuous batching over NetworkPools."""

    def __init__(self, pools: dict[str, NetworkPool], hbm_budget_bytes: int):
        self.pools = pools
        self.budget = int(hbm_budget_bytes)
        self.used = 0
        self.queue: deque = deque()

    def try_admit(self, now: float) -> None:
        """Admit queued requests in arrival order; a request whose network is
        full or that does not fit the budget waits, later requests for other
        networks may pass it."""
        waiting = deque()
        while self.queue:
            req = self.queue.popleft()
            pool = self.pools[req.network]
            need = pool.request_bytes(req)
            if pool.free and self.used + need <= self.budget:
                self.used += need
                pool.admit(req, now)
            else:
                waiting.append(req)
        self.queue = waiting

    def step(self, now: float, report: "ServeReport") -> bool:
        """One pass of the serving loop at time `now`: retire finished
        requests, admit queued ones, issue a tick on every pool that has work
        and room.  Returns whether any tick was issued."""
        for pool in self.pools.values():
            for req in pool.retire(now):
                self.used -= pool.request_bytes(req)
                report.requests.append(req)
        self.try_admit(now)
        issued = False
        for pool in self.pools.values():
            if pool.can_tick():
                pool.tick()
                issued = True
        return issued

    def run(self, requests: list[SimRequest], clock=time.perf_counter, idle_sleep: float = 50e-6,
            synchronize: bool = True) -> ServeReport:
        """Serve `requests` (their `arrival` times are seconds after start)."""
        for r in requests:
            pool = self.pools[r.network]
            st = r.stimulus
            if st.ndim != 2 or st.shape[0] < 1 or st.shape[1] != pool.c_in:
                raise ValueError(f"request {r.rid}: stimulus must be [steps >= 1, {pool.c_in}], got {tuple(st.shape)}")
            if pool.request_bytes(r) > self.budget:
                raise ValueError(f"request {r.rid} needs more device memory than the whole budget")
        arrivals = [(r.arrival, i, r) for i, r in enumerate(requests)]
        heapq.heapify(arrivals)
        report = ServeReport()
        t0 = clock()
        while arrivals or self.queue or any(p.busy() for p in self.pools.values()):
            now = clock() - t0
            while arrivals and arrivals[0][0] <= now:
                self.queue.append(heapq.heappop(arrivals)[2])
            if not self.step(now, report) and idle_sleep:
                time.sleep(idle_sleep)
        if synchronize:
            torch.cuda.synchronize()
        report.wall_s = clock() - t0
        report.events = sum(p.drain_events() for p in self.pools.values())
        report.ticks = {name: p.ticks for name, p in self.pools.items()}
        return report
