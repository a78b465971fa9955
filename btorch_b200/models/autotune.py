"""Autotuner of the fused engine's launch shapes.

The engine has three ways to deliver spikes (scatter over out-edges, ordered
gather over in-edges with a warp per neuron, sliced lane-per-neuron pull) and,
per way, tile parameters: samples per thread of the neuron launch and lanes
per active row in scatter, sample words per warp in pull.  Which is fastest
depends on the network (size, in-degree, delay range), the batch and the
activity, so the tuner times the candidates on the caller's own model and
input -- steps TRIAL_WARM .. TRIAL_WARM + TRIAL_STEPS of the call, run from
the caller's state, which is restored after every trial -- and caches the
winner on the model, keyed by the problem shape.  Candidates are limited to what the connection's sparse config
allows: "gather" (and `deterministic`) admits only the ordered gathers, whose
results are bit-identical to the reference's CPU product; "scatter" only
scatter; "auto" all three.

This replaces the reference's fixed Triton launch parameters
(btorch/_sparse_config.py:15-52, block_sources / edge_block / num_warps),
which a user had to pick by hand.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from .. import _lib as L
from .functional import named_hidden_states, set_hidden_states

TUNE_MIN_STEPS = 256   # calls shorter than this use the heuristic choice
TRIAL_WARM = 64        # steps run before the timed ones (activity ramps up from the initial state)
TRIAL_STEPS = 64       # steps timed per candidate


@dataclass(frozen=True)
class EngineChoice:
    mode: int                  # L.BT_MODE_*
    neuron_spt: int = 0        # scatter: samples per thread of the neuron launch (0 = default)
    scatter_lanes: int = 0     # scatter: lanes per active row, 8 or 32, or 1 = rows of a warp flattened
                               # into one edge range (0 = by mean row length)
    pull_words: int = 0        # pull: 32-sample mask words per warp (0 = one)
    dense_rows: int = -1       # scatter, one delay bin: spiking neurons from which a step is pulled
                               # densely (-1 = n / engine.DENSE_FRACTION, 0 = never)
    tile_posts: int = 0        # tile: posts per CTA (0 = one tile per SM); cluster: CTAs of the cluster (0 = most)

    def describe(self) -> dict:
        name = {L.BT_MODE_SCATTER: "scatter", L.BT_MODE_GATHER: "gather", L.BT_MODE_PULL: "pull",
                L.BT_MODE_TILE: "tile", L.BT_MODE_CLUSTER: "cluster"}[self.mode]
        return {"mode": name, "neuron_spt": self.neuron_spt, "scatter_lanes": self.scatter_lanes,
                "pull_words": self.pull_words, "dense_rows": self.dense_rows, "tile_posts": self.tile_posts}


def allowed_modes(conn, batch: int, receptors: int = 1, n_bins: int = 1) -> list[int]:
    """Delivery modes the sparse config admits (the sliced pull has no
    receptor channels: with receptors > 1 it is left out; the tile mode
    delivers push-wise like scatter, without delays or receptor channels; the
    cluster mode pulls like gather, without receptor channels, up to 32 delay
    bins)."""
    cfg = conn.sparse_config
    if cfg.deterministic or cfg.direction == "gather":
        modes = [L.BT_MODE_GATHER, L.BT_MODE_PULL]
    elif cfg.direction == "scatter":
        modes = [L.BT_MODE_SCATTER]
    else:
        modes = [L.BT_MODE_SCATTER, L.BT_MODE_PULL, L.BT_MODE_GATHER]
    if cfg.tile and cfg.direction != "gather" and not cfg.deterministic:
        # the persistent tile engine: opt-in -- its push delivery is slow in a
        # start-up burst, which the tuner's trial window (after a warm-up) misses
        modes.insert(1, L.BT_MODE_TILE)
    if cfg.direction != "scatter":
        # the single-cluster engine: an ordered in-edge gather (bit-exact, so
        # also under `deterministic`) for networks that fit one cluster's
        # shared memory, see candidates()
        modes.insert(1, L.BT_MODE_CLUSTER)
    modes = [m for m in modes if receptors == 1 or m != L.BT_MODE_PULL]
    if receptors > 1 or n_bins > 1 or batch > 256:
        modes = [m for m in modes if m != L.BT_MODE_TILE]
    if receptors > 1 or n_bins > 32 or batch > 256:
        modes = [m for m in modes if m != L.BT_MODE_CLUSTER]
    return modes


def heuristic(conn, batch: int, receptors: int = 1) -> EngineChoice:
    """The untuned choice: the configured direction (gather -> warp per neuron
    below `pull_min_batch` samples, sliced pull above; always warp per neuron
    with receptor channels), default tiles."""
    direction = conn.direction(batch)
    if direction == "gather":
        pull = batch >= conn.sparse_config.pull_min_batch and receptors == 1
        mode = L.BT_MODE_PULL if pull else L.BT_MODE_GATHER
    else:
        mode = L.BT_MODE_SCATTER
    return EngineChoice(mode)


def candidates(conn, batch: int, receptors: int = 1, n_bins: int = 1, n: int = 0, dev=None) -> list[EngineChoice]:
    out = []
    mw = L.lib().bt_mask_stride(batch)
    modes = allowed_modes(conn, batch, receptors, n_bins)
    for mode in modes:
        if mode == L.BT_MODE_CLUSTER:
            from .engine import cluster_shape, slices_of

            if n and dev is not None:
                lay = conn.engine_layout(1, 0, dev)
                slices_of(lay, dev)
                if cluster_shape(n, batch, lay.slices_ptr_host, n_bins=n_bins) is not None:
                    out.append(EngineChoice(mode))
            continue
        if mode == L.BT_MODE_TILE:
            from .engine import tile_shape

            base = tile_shape(n, batch, dev) if n and dev is not None else None
            if base is not None:
                for mult in (1, 2, 4):
                    tp = base[0] * mult
                    if mult > 1 and (tile_shape(n, batch, dev, tp) is None or -(-n // tp) < 8):
                        continue
                    out.append(EngineChoice(mode, tile_posts=0 if mult == 1 else tp))
            continue
        if mode == L.BT_MODE_SCATTER:
            for spt in (1, 2, 4):
                if spt > 1 and spt > batch:
                    continue
                for lanes in (1, 8, 32):
                    out.append(EngineChoice(mode, neuron_spt=spt, scatter_lanes=lanes))
        elif mode == L.BT_MODE_PULL:
            for words in sorted({1, mw} if mw in (2, 4) else {1}):
                out.append(EngineChoice(mode, pull_words=words))
        elif batch <= 32 or modes == [L.BT_MODE_GATHER]:  # a warp per neuron walks the samples serially
            out.append(EngineChoice(mode))
    return out


def _key(plan, batch: int, c_in: int) -> tuple:
    conn = plan.conn
    return (torch.cuda.get_device_name(plan.neuron.v.device), plan.neuron.size, batch, plan.n_bins,
            plan.uniform_delay, int(conn.indices.shape[1]), c_in, type(plan.neuron).__name__, plan.n_rec,
            tuple(allowed_modes(conn, batch, plan.n_rec, plan.n_bins)))


def tuned(rnn) -> dict:
    """Cached tuning results of `rnn`: key -> (choice, {choice: ms})."""
    return rnn.__dict__.setdefault("_bt_engine_tuning", {})


def choose(plan, rnn, x: torch.Tensor, sample_len, run) -> EngineChoice:
    """The engine choice for this call: cached, tuned now, or heuristic."""
    B = plan.neuron.v.reshape(-1, plan.neuron.size).shape[0]
    T = int(x.shape[0])
    c_in = int(x.shape[-1]) if plan.inp is not None else plan.neuron.size
    key = _key(plan, B, c_in)
    cache = tuned(rnn)
    if key in cache:
        return cache[key][0]
    if not plan.conn.sparse_config.autotune or T < TUNE_MIN_STEPS:
        return heuristic(plan.conn, B, plan.n_rec)
    cands = candidates(plan.conn, B, plan.n_rec, plan.n_bins, plan.neuron.size, plan.neuron.v.device)
    if plan.uniform_delay:  # a DelayedPSC delay: the tile mode has none
        cands = [c for c in cands if c.mode != L.BT_MODE_TILE]
    if len(cands) == 1:
        cache[key] = (cands[0], {})
        return cands[0]
    timings = {}
    state = {k: (v.detach().clone() if torch.is_tensor(v) else v) for k, v in named_hidden_states(rnn).items()}
    buffers = [(b, b.detach().clone()) for _, b in rnn.named_buffers()]
    graph, rnn.cudagraph = rnn.cudagraph, False
    dev = plan.neuron.v.device
    try:
        x_warm, x_timed = x[:TRIAL_WARM], x[TRIAL_WARM:TRIAL_WARM + TRIAL_STEPS]
        sl_timed = None if sample_len is None else (torch.as_tensor(sample_len) - TRIAL_WARM).clamp(min=0)
        for c in cands:
            for rep in range(2):  # first run builds layouts and warms up
                set_hidden_states(rnn, state, inplace=True)
                for b, v in buffers:
                    if not torch.equal(b, v):
                        b.copy_(v)
                run(plan, rnn, x_warm, sample_len=sample_len, choice=c)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(torch.cuda.current_stream(dev))
                run(plan, rnn, x_timed, sample_len=sl_timed, choice=c)
                e1.record(torch.cuda.current_stream(dev))
            torch.cuda.synchronize(dev)
            timings[c] = e0.elapsed_time(e1)
    finally:
        set_hidden_states(rnn, state, inplace=True)
        for b, v in buffers:
            if not torch.equal(b, v):
                b.copy_(v)
        rnn.cudagraph = graph
    best = min(timings, key=timings.get)
    cache[key] = (best, timings)
    return best
