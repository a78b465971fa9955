"""Benchmark of the B200 recurrent spiking step (one JSON line on rank 0).

Headline workload (--config batched): ALIF + exponential synapse (tau_syn
5 ms, adaptation tau 200 ms, dg_k 0.07), N = 65536 neurons, fixed in-degree
500 (32.8M fp32 weights), batch 64 samples with durations uniform in
[200, 2000] steps, Poisson input from 2000 channels at per-sample rates
uniform in [2, 40] Hz through a dense fp32 input layer, dt = 1 ms.  One bench
"step" simulates the whole batch (all 2000 time steps, finished samples
masked) through RecurrentNN's public forward, with CUDA-graph chunk replay.

Second workload (--config connectome, and by default appended to the
headline line as "connectome"): N = 140000 LIF neurons (c_m 64, tau 20,
refractory 2 ms, hard reset), lognormal in-degree (mean 350, sigma 1.0;
~49M synapses), weights = geometric synapse counts (mean 4) x +-2^-6 with the
sign by presynaptic type (70 % excitatory), per-synapse delays uniform in
1..20 steps (HeterSynapsePSC over the delay-expanded matrix), background
Poisson drive 8 x Poisson(0.25) per neuron and step (~11 Hz network rate),
batch 8, T = 2000.  Weights and drive are dyadic, so rasters are exact.  Its
object also carries the plain step: the same network at batch 1, launched
eagerly (no graph), on sample 0's input.

metric: synaptic events/s = sum over samples and time steps of the
out-degree of every neuron that spiked, divided by the device time.

--impl reference times the reference's CPU algorithm (the C oracle port of
btorch's native backend, all host threads) on a bounded sample of the same
workload.  Under torchrun every rank simulates its own batch (replicas,
weak scaling); the time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    "batched": dict(model="alif_dense_input", n=65536, indeg=500, batch=64, c_in=2000, t_max=2000,
                    rate=(2.0, 40.0), dur=(200, 2000), w_scale=0.0030, in_gain=1.0, s_state=36),
    "small": dict(model="alif_dense_input", n=65536, indeg=500, batch=64, c_in=2000, t_max=64,
                  rate=(2.0, 40.0), dur=(64, 64), w_scale=0.0030, in_gain=1.0, s_state=36),
    # s_state: v, psc, refractory r/w (24) + drive read (4) + delay-ring slot read and clear (8)
    "connectome": dict(model="lif_hetero_delay", n=140000, indeg=350, indeg_sigma=1.0, n_bins=20, exc=0.7,
                       batch=8, t_max=2000, dur=(2000, 2000), c_m=64.0, drive=(0.25, 8.0), s_state=36),
    # the connectome workload with receptor channels: HeterSynapsePSC(n_receptor=4), the (pre type, post
    # type) E/I pairs of make_hetersynapse_conn's neuron mode, a synaptic time constant per channel;
    # s_state: v, refractory r/w (16) + drive read (4) + per channel psc r/w and acc read/clear (16 C)
    "connectome_receptors": dict(model="lif_hetero_receptors", n=140000, indeg=350, indeg_sigma=1.0, n_bins=20,
                                 exc=0.7, batch=8, t_max=2000, dur=(2000, 2000), c_m=64.0, drive=(0.25, 8.0),
                                 receptors=4, taus=(5.0, 3.0, 10.0, 2.5), s_state=84),
    # shorter runs of the same workloads, for profiler captures (a few GB on the device)
    "batched_short": dict(model="alif_dense_input", n=65536, indeg=500, batch=64, c_in=2000, t_max=512,
                          rate=(2.0, 40.0), dur=(512, 512), w_scale=0.0030, in_gain=1.0, s_state=36),
    "connectome_short": dict(model="lif_hetero_delay", n=140000, indeg=350, indeg_sigma=1.0, n_bins=20, exc=0.7,
                             batch=8, t_max=256, dur=(256, 256), c_m=64.0, drive=(0.25, 8.0), s_state=36),
    "connectome_receptors_short": dict(model="lif_hetero_receptors", n=140000, indeg=350, indeg_sigma=1.0,
                                       n_bins=20, exc=0.7, batch=8, t_max=192, dur=(192, 192), c_m=64.0,
                                       drive=(0.25, 8.0), receptors=4, taus=(5.0, 3.0, 10.0, 2.5), s_state=84),
    # plain forward simulation: the reference's own CPU-runnable case, batch 1
    # (direction auto: the tuner picks among every delivery mode, the single-cluster engine included)
    "plain": dict(model="lif_plain", n=4096, p=0.02, batch=1, c_in=1000, t_max=1000, in_rate=0.01, in_std=0.05,
                  w_scale=0.1, dur=(1000, 1000), s_state=36, direction="auto"),
    # serving: Poisson request stream over a pool of connectome-shaped networks
    "serving": dict(model="serving", sizes=(16384, 32768, 65536, 140000), indeg=350, indeg_sigma=1.0, n_bins=20,
                    exc=0.7, c_m=64.0, c_in=4000, in_std=0.05, rate_hz=200.0, n_requests=200,
                    channels=(500, 4000), stim_hz=(5.0, 50.0), steps=(100, 5000), slots=16, chunk=128,
                    budget_gb=24.0),
    # truncated-BPTT training: windows of `window` steps, checkpointed chunks of `chunk`
    "training": dict(model="lif_train", n=8192, p=0.05, batch=128, t_max=500, window=100, chunk=20, unroll=10,
                     c_in=256, in_rate=0.02, in_std=0.1, w_exp=-9, inh_gain=6.0, n_out=10, alpha=5.0, lr=1e-3),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="batched", choices=sorted(CONFIGS))
    ap.add_argument("--extra", default="plain,connectome,connectome_receptors,training,serving",
                    help="comma-separated workloads measured after the headline one ('' for none)")
    ap.add_argument("--direction", default="scatter", choices=["scatter", "gather", "auto"])
    ap.add_argument("--no-cudagraph", action="store_true", help="launch every chunk eagerly")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=2, help="time steps per CPU-port sample")
    ap.add_argument("--cpu-events-steps", type=int, default=0,
                    help="reference arm: steps of the untimed event count (0 = the whole workload)")
    ap.add_argument("--no-parity", action="store_true", help="skip the parity checks against the oracle")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--ncu-window", type=int, default=None,
                    help="profile only time steps [S, S+64) (S a multiple of 64) of one extra batch after "
                         "the timed ones (cudaProfilerStart/Stop; use with ncu --profile-from-start off)")
    ap.add_argument("--engine-choice", default=None,
                    help="run the headline workload with this engine choice instead of the tuner's, e.g. "
                         "'scatter,spt=2,lanes=1' (profiling: the tuner's timings differ under a profiler)")
    return ap.parse_args()


def parse_choice(text):
    """'scatter,spt=2,lanes=1' / 'gather' / 'pull,words=2' / 'tile,tp=896' / 'cluster,ctas=8' -> autotune.EngineChoice."""
    if not text:
        return None
    from btorch_b200 import _lib as L
    from btorch_b200.models.autotune import EngineChoice

    mode, *kv = text.split(",")
    f = dict(item.split("=") for item in kv)
    modes = {"scatter": L.BT_MODE_SCATTER, "gather": L.BT_MODE_GATHER, "pull": L.BT_MODE_PULL,
             "tile": L.BT_MODE_TILE, "cluster": L.BT_MODE_CLUSTER}
    return EngineChoice(modes[mode], neuron_spt=int(f.get("spt", 0)), scatter_lanes=int(f.get("lanes", 0)),
                        pull_words=int(f.get("words", 0)), dense_rows=int(f.get("dense", -1)),
                        tile_posts=int(f.get("tp", f.get("ctas", 0))))


# ------------------------------------------------------------- workload --

def _dedupe_sorted(post, pre, n):
    key = post * n + pre
    key.sort()
    keep = np.ones(key.size, bool)
    keep[1:] = key[1:] != key[:-1]
    key = key[keep]
    return key // n, key % n


def make_network(cfg, seed=0):
    """dict(post, src, pre, w, n_bins, w_in): canonical (post, src) arrays; src
    is the presynaptic id, or pre * n_bins + delay bin for the delay-expanded
    matrix."""
    rng = np.random.default_rng(seed)
    n = cfg["n"]
    if cfg["model"] == "alif_dense_input":
        k = cfg["indeg"]
        src = rng.integers(0, n, size=(n, k), dtype=np.int64)
        src.sort(axis=1)
        for _ in range(50):
            dup = np.zeros_like(src, dtype=bool)
            dup[:, 1:] = src[:, 1:] == src[:, :-1]
            if not dup.any():
                break
            src[dup] = rng.integers(0, n, size=int(dup.sum()))
            src.sort(axis=1)
        post = np.repeat(np.arange(n, dtype=np.int64), k)
        src = src.reshape(-1)
        exc = src < int(0.8 * n)
        w = rng.lognormal(-1.0, 1.0, size=src.size).astype(np.float32) * np.float32(cfg["w_scale"])
        w = np.where(exc, w, np.float32(-0.4) * w).astype(np.float32)
        w_in = (rng.normal(0.0, 0.05, size=(cfg["c_in"], n)) * cfg["in_gain"]).astype(np.float32)
        return dict(post=post, src=src, pre=src, w=w, n_bins=1, w_in=w_in)
    if cfg["model"] == "lif_plain":
        # fixed connection probability (binomial in-degree), lognormal weights,
        # inhibitory presynaptic neurons (last 20 %) scaled by -0.4
        k = rng.binomial(n, cfg["p"], size=n)
        post = np.repeat(np.arange(n, dtype=np.int64), k)
        pre = rng.integers(0, n, size=post.size, dtype=np.int64)
        post, pre = _dedupe_sorted(post, pre, n)
        w = rng.lognormal(-1.0, 1.0, size=pre.size).astype(np.float32) * np.float32(cfg["w_scale"])
        w = np.where(pre < int(0.8 * n), w, np.float32(-0.4) * w).astype(np.float32)
        w_in = rng.normal(0.0, cfg["in_std"], size=(cfg["c_in"], n)).astype(np.float32)
        return dict(post=post, src=pre, pre=pre, w=w, n_bins=1, w_in=w_in)
    # connectome-shaped: lognormal in-degree, presynaptic type sets the sign,
    # per-synapse delay d in 1..R lands in delay bin d - 1
    R = cfg["n_bins"]
    sigma = cfg["indeg_sigma"]
    mu = np.log(cfg["indeg"]) - sigma ** 2 / 2
    k = np.clip(np.rint(rng.lognormal(mu, sigma, n)), 1, n - 1).astype(np.int64)
    post = np.repeat(np.arange(n, dtype=np.int64), k)
    pre = rng.integers(0, n, size=post.size, dtype=np.int64)
    post, pre = _dedupe_sorted(post, pre, n)
    delay = rng.integers(1, R + 1, size=post.size)
    count = rng.geometric(0.25, size=post.size)
    w = (count * np.where(pre < int(cfg["exc"] * n), 1.0, -1.0) * 2.0 ** -6).astype(np.float32)
    src = pre * R + (delay - 1)
    C = cfg.get("receptors", 1)
    if C > 1:
        # column post * 4 + pair, pair = 2 type(pre) + type(post), type 0 = E (the first exc * n ids), 1 = I:
        # the stacked layout of make_hetersynapse_conn's neuron mode; re-sorted into (column, src) order
        inh = np.arange(n) >= int(cfg["exc"] * n)
        col = post * C + 2 * inh[pre] + inh[post]
        order = np.lexsort((src, col))
        post, src, pre, delay, w = col[order], src[order], pre[order], delay[order], w[order]
    return dict(post=post, src=src, pre=pre, delay_bin=delay - 1, w=w, n_bins=R, w_in=None, n_rec=C)


def make_training_network(cfg, seed=0):
    """Fixed-probability recurrent net (binomial in-degree), dyadic weights:
    geometric synapse counts x 2^w_exp, inhibitory (last 20 % of presynaptic
    ids) x -inh_gain; dense input weights N(0, in_std); readout targets are 10
    sinusoids per sample (frequency U[1, 20] Hz, phase U[0, 2 pi))."""
    rng = np.random.default_rng(seed)
    n = cfg["n"]
    k = rng.binomial(n, cfg["p"], size=n)
    post = np.repeat(np.arange(n, dtype=np.int64), k)
    pre = rng.integers(0, n, size=post.size, dtype=np.int64)
    post, pre = _dedupe_sorted(post, pre, n)
    count = rng.geometric(0.25, size=post.size)
    w = (count * np.where(pre < int(0.8 * n), 1.0, -cfg["inh_gain"]) * 2.0 ** cfg["w_exp"]).astype(np.float32)
    w_in = rng.normal(0.0, cfg["in_std"], size=(cfg["c_in"], n)).astype(np.float32)
    T, B, m = cfg["t_max"], cfg["batch"], cfg["n_out"]
    freq = rng.uniform(1.0, 20.0, size=(1, B, m))
    phase = rng.uniform(0.0, 2 * np.pi, size=(1, B, m))
    target = np.sin(2 * np.pi * freq * np.arange(T)[:, None, None] * 1e-3 + phase).astype(np.float32)
    return dict(post=post, src=pre, pre=pre, w=w, n_bins=1, w_in=w_in, target=target)


def measure_training(cfg, args, dev):
    """Truncated BPTT on the training workload: per window, forward through
    the fused BPTT (one autograd Function over the hand-written forward and
    backward kernels, input projection included; with grad_checkpoint the
    forward keeps the state at every chunk start and the backward recomputes
    each chunk of `chunk` steps), readout + MSE, backward, Adam step,
    detach_net.  Returns the sub-object of the JSON line (forward synaptic
    events per second of training time, windows per second)."""
    from btorch_b200.models import LIF, DenseConn, ExponentialPSC, RecurrentNN, Sigmoid, SparseConn, environ
    from btorch_b200.models.functional import detach_net, init_net_state

    net = make_training_network(cfg, args.seed)
    n, B, Wn = cfg["n"], cfg["batch"], cfg["window"]
    conn = SparseConn.from_canonical(net["post"], net["src"], net["w"], (n, n), enforce_dale=False,
                                     sparse_config={"direction": args.direction})
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True,
                 surrogate_function=Sigmoid(alpha=cfg["alpha"]))
    brain = RecurrentNN(neuron, ExponentialPSC(n, tau_syn=5.0, linear=conn),
                        neuron_inp_module=DenseConn(cfg["c_in"], n, weight=torch.from_numpy(net["w_in"])),
                        update_state_names=(), grad_checkpoint=True, chunk_size=cfg["chunk"],
                        unroll=cfg["unroll"]).to(dev)
    readout = torch.nn.Linear(n, cfg["n_out"]).to(dev)
    opt = torch.optim.Adam(list(brain.parameters()) + list(readout.parameters()), lr=cfg["lr"])
    import torch.distributed as dist

    from btorch_b200.replicas import allreduce_gradients

    world = dist.get_world_size() if dist.is_initialized() else 1
    rank = dist.get_rank() if dist.is_initialized() else 0
    params = list(brain.parameters()) + list(readout.parameters())
    g = torch.Generator(device=dev).manual_seed(20_000 + args.seed + rank)  # each replica its own samples
    x = torch.poisson(torch.full((cfg["t_max"], B, cfg["c_in"]), cfg["in_rate"], device=dev), generator=g)
    target = torch.from_numpy(net["target"]).to(dev)
    outdeg = torch.bincount(torch.from_numpy(net["pre"]), minlength=n).to(dev, torch.float64)
    n_win = cfg["t_max"] // Wn
    losses = []

    def window(k, events=None):
        sl = slice((k % n_win) * Wn, (k % n_win + 1) * Wn)
        if k % n_win == 0:
            init_net_state(brain, batch_size=B, dtype=torch.float32, device=dev)
        with environ.context(dt=1.0):
            z, _ = brain(x[sl])
            loss = ((readout(z) - target[sl]) ** 2).mean()
            opt.zero_grad(set_to_none=True)
            loss.backward()
            # data parallel over replicas: one all-reduce of every gradient
            allreduce_gradients(params)
            opt.step()
        detach_net(brain)
        if events is not None:
            events.append((z.detach().sum(dim=(0, 1)).double() * outdeg).sum())
            losses.append(loss.detach())

    for k in range(max(3, args.warmup)):
        window(k)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    events = []
    steps = max(args.steps, 1) * n_win
    e0.record(stream)
    for k in range(steps):
        window(k, events)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ev = float(torch.stack(events).sum())
    if world > 1:
        ms, ev = job_totals(ms, ev, dev)
    return {"value": ev / (ms * 1e-3), "unit": "forward synaptic events/s of training time",
            "replicas": world, "gradient_allreduce_bytes_per_step": 4 * sum(p.numel() for p in params)
            if world > 1 else 0,
            "ms_per_window": ms / steps, "windows": steps, "window_steps": Wn,
            "neuron_steps_per_s": n * B * Wn * steps * world / (ms * 1e-3),
            "loss_first_last": [float(losses[0]), float(losses[-1])], "direction": conn.direction(B),
            "path": brain.last_path, "bptt": getattr(brain, "last_bptt", None),
            "config": {"workload": f"training: LIF+ExpPSC N={n} p={cfg['p']} ({len(net['w'])} trainable weights) "
                                   f"batch {B} T {cfg['t_max']} TBPTT windows {Wn} checkpoint chunks "
                                   f"{cfg['chunk']} (recomputed in backward) sigmoid alpha {cfg['alpha']} "
                                   f"readout {cfg['n_out']} sinusoids, MSE, Adam"}}


def measure_serving(cfg, args, dev):
    """Continuous batching (btorch_b200.serving) of a seeded Poisson request
    stream over four connectome-shaped networks (the connectome generator at
    each size, plus a dense input layer of c_in channels with half-normal
    weights).  Each request drives a random number of channels at its own
    rate for its own number of steps; stimuli are synthesised on the device
    before the run (they stand in for client uploads).

    Three load points: the configured arrival rate (200 req/s, above what the
    server sustains: its latency is mostly queueing), then the server's
    capacity measured there (requests completed per second) and the same
    request mix offered at 50 % and 90 % of it.  Each reports p50/p99 latency
    (arrival to completion) and wait (arrival to admission), the latter also
    in ticks of the slowest network (one tick = `chunk` steps of all its
    slots, timed alone with every slot busy)."""
    from btorch_b200.models import DenseConn
    from btorch_b200.serving import NetworkPool, SimRequest, SimulationServer

    pools = {}
    rng = np.random.default_rng(30_000 + args.seed)
    for i, n in enumerate(cfg["sizes"]):
        ncfg = dict(CONFIGS["connectome"], n=n, batch=cfg["slots"])
        net = make_network(ncfg, args.seed + i)
        rnn = build_model(ncfg, net, dev, args.direction)
        w_in = np.abs(rng.normal(0.0, cfg["in_std"], size=(cfg["c_in"], n))).astype(np.float32)
        w_in = (np.round(w_in * 256.0) / 256.0).astype(np.float32)  # dyadic: exact sums
        rnn.neuron_inp_module = DenseConn(cfg["c_in"], n, weight=torch.from_numpy(w_in)).to(dev)
        pools[f"n{n}"] = NetworkPool(f"n{n}", rnn, slots=cfg["slots"], chunk=cfg["chunk"], device=dev)
    names = list(pools)
    g = torch.Generator(device=dev).manual_seed(40_000 + args.seed)
    mix = []  # (gap in units of the mean inter-arrival time, network, stimulus)
    for i in range(cfg["n_requests"]):
        gap = rng.exponential(1.0)
        T = int(rng.integers(cfg["steps"][0], cfg["steps"][1] + 1))
        c = int(rng.integers(cfg["channels"][0], cfg["channels"][1] + 1))
        hz = float(rng.uniform(*cfg["stim_hz"]))
        stim = torch.zeros((T, cfg["c_in"]), device=dev)
        stim[:, :c] = torch.poisson(torch.full((T, c), hz * 1e-3, device=dev), generator=g)
        mix.append((gap, names[int(rng.integers(len(names)))], stim))

    def requests(rate):
        t, out = 0.0, []
        for i, (gap, name, stim) in enumerate(mix):
            t += gap / rate
            out.append(SimRequest(network=name, stimulus=stim, arrival=t, rid=i))
        return out

    # warm-up: one tick per pool (graph capture) outside the measured runs,
    # then each pool's tick time alone with every slot busy
    warm = [SimRequest(network=nm, stimulus=torch.zeros((p.chunk, cfg["c_in"]), device=dev), rid=-1 - j)
            for j, (nm, p) in enumerate(pools.items())]
    SimulationServer(pools, hbm_budget_bytes=int(cfg["budget_gb"] * 2**30)).run(warm)
    tick_ms = {}
    for nm, p in pools.items():
        full = [SimRequest(network=nm, stimulus=torch.zeros((p.chunk * 3, cfg["c_in"]), device=dev), rid=-100 - s)
                for s in range(p.slots)]
        t0 = time.perf_counter()
        SimulationServer({nm: p}, hbm_budget_bytes=int(cfg["budget_gb"] * 2**30)).run(full)
        tick_ms[nm] = (time.perf_counter() - t0) * 1e3 / 3
    tick = max(tick_ms.values())

    def serve(rate):
        for p in pools.values():
            p.drain_events()
            p.events = 0
            p.ticks = 0
        server = SimulationServer(pools, hbm_budget_bytes=int(cfg["budget_gb"] * 2**30))
        rep = server.run(requests(rate))
        out = rep.summary()
        lat = np.array([r.latency for r in rep.requests]) * 1e3
        wait = np.array([r.t_admit - r.arrival for r in rep.requests]) * 1e3
        steps = sum(r.steps for r in rep.requests)
        out.update({"offered_rate_req_per_s": rate, "completed_req_per_s": len(rep.requests) / rep.wall_s,
                    "mean_latency_ms": float(lat.mean()), "p50_wait_ms": float(np.percentile(wait, 50)),
                    "p99_wait_ms": float(np.percentile(wait, 99)),
                    "p99_wait_ticks": float(np.percentile(wait, 99)) / tick,
                    "sample_steps_per_s": steps / rep.wall_s})
        return out

    out = serve(cfg["rate_hz"])
    capacity = out["completed_req_per_s"]
    out["load_points"] = {"saturated": {k: out[k] for k in ("offered_rate_req_per_s", "completed_req_per_s", "p50_ms",
                                                             "p99_ms", "p50_wait_ms", "p99_wait_ms",
                                                             "p99_wait_ticks")}}
    for frac in (0.5, 0.9):
        r = serve(frac * capacity)
        out["load_points"][f"{int(frac * 100)}pct_of_capacity"] = {
            k: r[k] for k in ("offered_rate_req_per_s", "completed_req_per_s", "p50_ms", "p99_ms", "p50_wait_ms",
                              "p99_wait_ms", "p99_wait_ticks", "events_per_s")}
    out.update({"unit": "ms (latency), events/s", "capacity_req_per_s": capacity, "tick_ms_alone": tick_ms,
                "direction": args.direction,
                "config": {"workload": f"serving: {cfg['n_requests']} requests, Poisson arrivals "
                                       f"{cfg['rate_hz']} req/s (and 50 %, 90 % of the measured capacity) over "
                                       f"networks N={list(cfg['sizes'])} (connectome-shaped, delays "
                                       f"1..{cfg['n_bins']}), {cfg['slots']} slots each, ticks of "
                                       f"{[p.chunk for p in pools.values()]} steps, stimulus {cfg['channels']} "
                                       f"channels at {cfg['stim_hz']} Hz for {cfg['steps']} steps, HBM budget "
                                       f"{cfg['budget_gb']} GiB"}})
    return out


def build_model(cfg, net, device, direction, batch=None):
    import pandas as pd

    from btorch_b200.models import (ALIF, LIF, DenseConn, ExponentialPSC, HeterSynapsePSC, RecurrentNN,
                                    SparseConn)
    from btorch_b200.models.functional import init_net_state

    n, R, C = cfg["n"], net["n_bins"], net.get("n_rec", 1)
    conn = SparseConn.from_canonical(net["post"], net["src"], net["w"], (n * R, n * C), enforce_dale=False,
                                     sparse_config={"direction": direction})
    if cfg["model"] == "alif_dense_input":
        neuron = ALIF(n, v_threshold=1.0, v_reset=0.0, c_m=1.0, g_leak=0.05, E_leak=0.0, E_k=-1.0,
                      tau_adapt=200.0, dg_k=0.07, tau_ref=2.0, hard_reset=True)
        syn = ExponentialPSC(n, tau_syn=5.0, linear=conn)
        inp = DenseConn(cfg["c_in"], n, weight=torch.from_numpy(net["w_in"]))
    elif cfg["model"] == "lif_plain":
        neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True)
        syn = ExponentialPSC(n, tau_syn=5.0, linear=conn)
        inp = DenseConn(cfg["c_in"], n, weight=torch.from_numpy(net["w_in"]))
    elif C > 1:
        neuron = LIF(n, v_threshold=1.0, v_reset=0.0, c_m=cfg["c_m"], tau=20.0, tau_ref=2.0, hard_reset=True)
        rti = pd.DataFrame([(0, "E", "E"), (1, "E", "I"), (2, "I", "E"), (3, "I", "I")],
                           columns=["receptor_index", "pre_receptor_type", "post_receptor_type"])
        taus = torch.tensor(cfg["taus"], dtype=torch.float32).repeat(n)
        syn = HeterSynapsePSC(n, C, rti, conn, base_psc=ExponentialPSC, max_delay_steps=R,
                              use_circular_buffer=True, tau_syn=taus)
        inp = None
    else:
        neuron = LIF(n, v_threshold=1.0, v_reset=0.0, c_m=cfg["c_m"], tau=20.0, tau_ref=2.0, hard_reset=True)
        rti = pd.DataFrame({"receptor_type": ["syn"], "receptor_index": [0]})
        syn = HeterSynapsePSC(n, 1, rti, conn, base_psc=ExponentialPSC, max_delay_steps=R,
                              use_circular_buffer=True, tau_syn=5.0)
        inp = None
    rnn = RecurrentNN(neuron, syn, neuron_inp_module=inp, update_state_names=()).to(device)
    init_net_state(rnn, batch_size=batch or cfg["batch"], dtype=torch.float32, device=device)
    return rnn


def make_inputs(cfg, seed, device):
    g = torch.Generator(device=device).manual_seed(10_000 + seed)
    B, T = cfg["batch"], cfg["t_max"]
    if cfg["model"] == "alif_dense_input":
        C = cfg["c_in"]
        lo, hi = cfg["rate"]
        rates = lo + (hi - lo) * torch.rand(B, generator=g, device=device)
        p = (rates * 1e-3).view(1, B, 1).expand(T, B, C)
        x = torch.poisson(p.contiguous(), generator=g)
    elif cfg["model"] == "lif_plain":
        x = torch.poisson(torch.full((T, B, cfg["c_in"]), cfg["in_rate"], device=device), generator=g)
    else:
        lam, amp = cfg["drive"]
        x = torch.empty((T, B, cfg["n"]), device=device, dtype=torch.float32)
        rate = torch.full((B, cfg["n"]), lam, device=device)
        for t in range(T):
            x[t] = torch.poisson(rate, generator=g) * amp
    dlo, dhi = cfg["dur"]
    lens = torch.randint(dlo, dhi + 1, (B,), generator=g, device=device)
    return x, lens


def describe(name, cfg):
    if cfg["model"] == "lif_plain":
        return (f"{name}: LIF+ExpPSC N={cfg['n']} p={cfg['p']} lognormal(-1,1)x{cfg['w_scale']} E/I 80/20 "
                f"batch {cfg['batch']} T {cfg['t_max']} c_in {cfg['c_in']} at {cfg['in_rate'] * 1e3:.0f} Hz")
    if cfg["model"] == "alif_dense_input":
        return (f"{name}: ALIF+ExpPSC N={cfg['n']} fixed in-degree {cfg['indeg']} batch {cfg['batch']} "
                f"durations {cfg['dur']} T_max {cfg['t_max']} c_in {cfg['c_in']}")
    rec = (f" {cfg['receptors']} receptor channels (E/I pairs, tau_syn {'/'.join(map(str, cfg['taus']))})"
           if cfg.get("receptors", 1) > 1 else "")
    return (f"{name}: LIF+HeterSynapsePSC(ExpPSC) N={cfg['n']} lognormal in-degree mean {cfg['indeg']} "
            f"sigma {cfg['indeg_sigma']} delays 1..{cfg['n_bins']}{rec} batch {cfg['batch']} T {cfg['t_max']} "
            f"drive {cfg['drive'][1]} x Poisson({cfg['drive'][0]})")


# --------------------------------------------------------------- clocks --

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        load = [s for s in sm if smax and s > 0.3 * max(smax)] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows)}


# -------------------------------------------------------------- oracle --

def oracle_spec(cfg, net):
    from oracle import oracle as O

    n = cfg["n"]
    ptr = np.zeros(n + 1, np.int64)
    ptr[1:] = np.cumsum(np.bincount(net["post"], minlength=n))
    lin = -1.0 / torch.as_tensor(5.0)
    coef_syn = float(torch.expm1(1.0 * lin) / lin)
    if cfg["model"] == "alif_dense_input":
        lin = -1.0 / torch.as_tensor(200.0)
        coef_gk = float(torch.expm1(1.0 * lin) / lin)
        params = {"v_threshold": 1.0, "v_reset": 0.0, "c_m": 1.0, "g_leak": 0.05, "E_leak": 0.0, "E_k": -1.0,
                  "dg_k": 0.07, "tau_adapt": 200.0, "coef_gk": coef_gk, "tau_ref": 2.0, "psc_coef": coef_syn,
                  "psc_tau": 5.0}
        return O.NetSpec(n=n, kind=1, hard_reset=True, use_ref=True, dt=1.0, params=params, ptr=ptr,
                         pre=net["pre"].astype(np.int32), delay=np.zeros(net["pre"].size, np.int32), w=net["w"])
    if cfg["model"] == "lif_plain":
        params = {"v_threshold": 1.0, "v_reset": 0.0, "c_m": 1.0, "tau": 20.0, "tau_ref": 2.0,
                  "psc_coef": coef_syn, "psc_tau": 5.0}
        return O.NetSpec(n=n, kind=0, hard_reset=True, use_ref=True, dt=1.0, params=params, ptr=ptr,
                         pre=net["pre"].astype(np.int32), delay=np.zeros(net["pre"].size, np.int32), w=net["w"])
    params = {"v_threshold": 1.0, "v_reset": 0.0, "c_m": cfg["c_m"], "tau": 20.0, "tau_ref": 2.0,
              "psc_coef": coef_syn, "psc_tau": 5.0}
    return O.NetSpec(n=n, kind=0, hard_reset=True, use_ref=True, dt=1.0, params=params, ptr=ptr,
                     pre=net["pre"].astype(np.int32), delay=net["delay_bin"].astype(np.int32), w=net["w"],
                     max_delay=net["n_bins"] - 1)


class CpuPort:
    """The oracle's port of the reference's CPU step -- every synapse every
    step, as torch.sparse.mm computes it, and the dense input layer's
    projection -- on all host threads, its state carried from one sample of
    time steps to the next (so a sample can start past the start-up burst)."""

    def __init__(self, cfg, net, batch):
        from oracle import oracle as O

        self.O = O
        self.cfg, self.net = cfg, net
        self.spec = oracle_spec(cfg, net)
        self.state = O.init_state(self.spec, batch)
        self.threads = os.cpu_count() or 1
        self.outdeg = np.bincount(net["pre"], minlength=cfg["n"]).astype(np.int64)
        self.steps = 0

    def advance(self, x_cpu):
        """Run len(x_cpu) steps; returns (synaptic events, seconds, spikes uint8 [S, B, n])."""
        S, B = x_cpu.shape[:2]
        t0 = time.perf_counter()
        if self.net["w_in"] is not None:
            xp = self.O.linear_t(x_cpu.reshape(S * B, -1), self.net["w_in"], threads=self.threads).reshape(S, B, -1)
        else:
            xp = x_cpu
        out = self.O.run(self.spec, self.state, xp, threads=self.threads)
        dt = time.perf_counter() - t0
        self.steps += S
        events = int((out["spikes"].astype(np.int64) * self.outdeg[None, None, :]).sum())
        return events, dt, out["spikes"]


def cpu_sample(cfg, net, x_cpu, steps):
    """The port on the first `steps` time steps of the batch from rest;
    returns (events, seconds, threads, spikes)."""
    port = CpuPort(cfg, net, x_cpu.shape[1])
    e, t, z = port.advance(x_cpu[:steps])
    return e, t, port.threads, z


def host_inputs(cfg, seed, steps):
    """Seeded host-side input of the workload's shape for `steps` steps and
    the samples' durations (the reference arm has no GPU): per-sample Poisson
    rates over the input channels, or the background drive."""
    rng = np.random.default_rng(10_000 + seed)
    B = cfg["batch"]
    if cfg["model"] in ("alif_dense_input",):
        rates = rng.uniform(*cfg["rate"], size=B)
        x = rng.poisson(np.broadcast_to((rates * 1e-3)[None, :, None], (steps, B, cfg["c_in"]))).astype(np.float32)
    elif cfg["model"] == "lif_plain":
        x = rng.poisson(cfg["in_rate"], (steps, B, cfg["c_in"])).astype(np.float32)
    else:
        lam, amp = cfg["drive"]
        x = (rng.poisson(lam, (steps, B, cfg["n"])) * amp).astype(np.float32)
    lens = rng.integers(cfg["dur"][0], cfg["dur"][1] + 1, B)
    return x, lens


def workload_events(cfg, net, x_host, lens, chunk=128):
    """Synaptic events of the whole batch (every sample to its length) and
    its live sample-steps, from the oracle's event-driven run (bit-identical
    to the reference's; untimed), chunk by chunk so that the projected input
    never holds more than `chunk` steps."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    spec = oracle_spec(cfg, net)
    T, B = x_host.shape[:2]
    st = O.init_state(spec, B)
    outdeg = np.bincount(net["pre"], minlength=cfg["n"]).astype(np.int64)
    lens = np.minimum(np.asarray(lens), T)
    events = 0
    for k0 in range(0, int(lens.max()), chunk):
        kc = min(chunk, T - k0)
        xc = x_host[k0:k0 + kc]
        if net["w_in"] is not None:
            xc = O.linear_t(xc.reshape(kc * B, -1), net["w_in"], threads=threads).reshape(kc, B, -1)
        out = O.run(spec, st, xc, sample_len=np.clip(lens - k0, 0, kc).astype(np.int32), threads=threads,
                    events=True)
        events += int((out["spikes"].astype(np.int64) * outdeg[None, None, :]).sum())
    return events, int(lens.sum())


def cpu_throughput(events_per_sample_step, seconds, sample_steps):
    """events/s of the CPU port on the whole workload: its measured time per
    live sample-step (the port's cost per step does not depend on the
    activity: every synapse is visited) times the workload's mean events per
    live sample-step."""
    return events_per_sample_step * sample_steps / seconds


# -------------------------------------------------------------- parity --
#
# The checker: the engine on the configurations' own networks and inputs at
# their full sizes, against the oracle (event-driven push, bit-identical to
# the reference's per-synapse chain), outside every timed region.


def raster_bits(raster, n):
    """[T, B, ceil(n/32)] int32 bitmask raster (device or host) -> uint8 [T, B, n]."""
    r = raster.cpu().numpy() if torch.is_tensor(raster) else raster
    return np.unpackbits(np.ascontiguousarray(r).view(np.uint8), axis=-1, bitorder="little")[..., :n]


def engine_window(cfg, net, x, lens, dev, direction, steps, trace_v=False, cudagraph=True, choice=None):
    """A fresh model of the workload run for `steps` steps on x[:steps]
    (`choice`: a parse_choice string pinning the delivery mode, else the
    tuner's).  Returns (spikes uint8 [steps, B, n], final state dict of numpy
    arrays, v trace or None, the model's delivery direction and mode)."""
    from btorch_b200.models import environ
    from btorch_b200.models import engine as E

    rnn = build_model(cfg, net, dev, direction)
    rnn.cudagraph = cudagraph
    if trace_v:
        rnn.update_state_names = ("neuron.v",)
    sl = None if lens is None else lens.clamp(max=steps)
    with torch.inference_mode(), environ.context(dt=1.0):
        raster, st = rnn(x[:steps].contiguous(), sample_len=sl, spikes_out="bitmask",
                         engine_choice=parse_choice(choice))
    plan, _ = E.match(rnn)
    final = {"v": rnn.neuron.v, "psc": plan.psc_mod.psc, "ref": rnn.neuron.refractory}
    if cfg["model"] == "alif_dense_input":
        final["gk"] = rnn.neuron.g_k
    final = {k: t.reshape(t.shape[0], -1).cpu().numpy() for k, t in final.items()}
    vtr = st["neuron.v"].cpu().numpy() if trace_v else None
    direction = f"{rnn.last_engine_direction} ({rnn.last_engine_choice.describe()['mode']})"
    del rnn
    return raster_bits(raster, cfg["n"]), final, vtr, direction


def oracle_window(cfg, net, x_host, steps, lens=None, trace_v=False):
    """The oracle over the same steps (event-driven push; the projection of a
    dense input layer as the ascending-channel chain the engine uses)."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    spec = oracle_spec(cfg, net)
    B = x_host.shape[1]
    if net["w_in"] is not None:
        xp = O.linear_t(x_host[:steps].reshape(steps * B, -1), net["w_in"], threads=threads).reshape(steps, B, -1)
    else:
        xp = x_host[:steps]
    st = O.init_state(spec, B)
    sl = None if lens is None else np.minimum(np.asarray(lens), steps).astype(np.int32)
    out = O.run(spec, st, xp, sample_len=sl, threads=threads, want_v=trace_v, events=True)
    final = {"v": st.v, "psc": st.psc, "ref": st.ref}
    if spec.kind == 1:
        final["gk"] = st.gk
    return out["spikes"], final, out["v"]


def first_divergence(a, b):
    """First step at which two [T, B, n] rasters differ (T if never)."""
    bad = np.nonzero((a != b).reshape(len(a), -1).any(1))[0]
    return int(bad[0]) if bad.size else len(a)


def _sample_divergence(a, b):
    """Per sample: the first step at which its rasters differ (T if never)."""
    T, B = a.shape[:2]
    bad = (a != b).any(-1)  # [T, B]
    return np.where(bad.any(0), bad.argmax(0), T)


def parity_bitwise(name, cfg, net, x, lens, dev, steps, direction, choice=None):
    """Rasters of every step and the final state bit for bit (dyadic
    weights, or an ordered delivery mode)."""
    t0 = time.perf_counter()
    z, fin, _, used = engine_window(cfg, net, x, lens, dev, direction, steps, choice=choice)
    oz, ofin, _ = oracle_window(cfg, net, x.cpu().numpy() if torch.is_tensor(x) else x, steps,
                                None if lens is None else lens.cpu().numpy())
    k = first_divergence(z, oz)
    state_equal = {key: bool(np.array_equal(fin[key], ofin[key])) for key in ofin if ofin[key] is not None}
    ok = k == steps and all(state_equal.values())
    return {"check": "bitwise" if ok else "MISMATCH", "steps": steps, "direction": used,
            "rasters_equal_steps": k, "final_state_equal": state_equal, "spikes": int(oz.sum()),
            "seconds": round(time.perf_counter() - t0, 1)}


def parity_tolerance(name, cfg, net, x, lens, dev, steps, direction, rtol=1e-5):
    """Non-dyadic weights summed in arrival order: per sample, the raster
    equal and v within rel `rtol` (atol rtol) of the oracle until that
    sample's first spike divergence."""
    t0 = time.perf_counter()
    z, _, vtr, used = engine_window(cfg, net, x, lens, dev, direction, steps, trace_v=True)
    oz, _, ov = oracle_window(cfg, net, x.cpu().numpy() if torch.is_tensor(x) else x, steps,
                              None if lens is None else lens.cpu().numpy(), trace_v=True)
    ks = _sample_divergence(z, oz)
    used_tol = max_abs = 0.0
    for b, k in enumerate(ks):
        if k == 0:
            continue
        a, r = vtr[:k, b].astype(np.float64), ov[:k, b].astype(np.float64)
        d = np.abs(a - r)
        max_abs = max(max_abs, float(d.max()))
        used_tol = max(used_tol, float((d / (rtol * np.abs(r) + rtol)).max()))  # <= 1: within tolerance
    ok = used_tol <= 1.0 and bool(ks.min() >= 1)
    return {"check": f"within rel {rtol:g} (atol {rtol:g}) until divergence" if ok else "MISMATCH",
            "steps": steps, "direction": used, "first_divergence": int(ks.min()),
            "median_sample_divergence": float(np.median(ks)), "samples_never_diverged": int((ks == steps).sum()),
            "max_abs_err_before_divergence": max_abs, "tolerance_used": used_tol, "spikes": int(oz.sum()),
            "seconds": round(time.perf_counter() - t0, 1)}


# ---------------------------------------------------------------- main --

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def reference_arm(args, cfg, world, rank):
    """The reference's CPU algorithm (the oracle's port of btorch's native
    backend: torch.sparse.mm over every synapse each step, eager neuron and
    synapse updates, the dense input layer), on all host threads.

    The port's cost per step is the same whatever the activity, while the
    workload's events are concentrated in its start-up burst, so events/s is
    taken as whole-workload events (counted once, untimed, by the oracle's
    event-driven run, which gives the same raster) per live sample-step,
    times the port's measured live sample-steps per second.  Each bench step
    times --cpu-sample-steps time steps of the whole batch, continuing the
    simulation from the previous one.  The reference package itself cannot be
    installed here (its build backend is not in the offline wheel set), so
    its own modules do not run on this host."""
    if rank != 0:
        return
    net = make_network(cfg, args.seed)
    S = args.cpu_sample_steps
    B = cfg["batch"]
    T = cfg["t_max"] if not args.cpu_events_steps else min(cfg["t_max"], args.cpu_events_steps)
    x, lens = host_inputs(cfg, args.seed, max(T, (args.warmup + args.steps) * S))
    t0 = time.perf_counter()
    ev_total, sample_steps = workload_events(cfg, net, x[:T], lens)
    count_s = time.perf_counter() - t0
    eps = ev_total / sample_steps
    port = CpuPort(cfg, net, B)
    k = 0
    for _ in range(args.warmup):
        port.advance(x[k:k + S])
        k += S
    tot_t = 0.0
    for _ in range(args.steps):
        _, t, _ = port.advance(x[k:k + S])
        k += S
        tot_t += t
    val = cpu_throughput(eps, tot_t, args.steps * S * B)
    sample = (f"{S} time steps of the {B}-sample batch per step (port, timed); whole-workload events per live "
              f"sample-step {eps:.4g} from an untimed event-driven run of {T} steps ({count_s:.0f} s)")
    line = {"metric": "synaptic_events_per_s", "value": val, "unit": "events/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": describe(args.config, cfg), "parallelism": "replicas"},
            "neuron_steps_per_s": cfg["n"] * B * S * args.steps / tot_t,
            "cpu_baseline": {"value": val, "unit": "events/s", "cores": port.threads, "kind": "port",
                             "sample": sample,
                             "note": "the reference package cannot be installed offline (build backend hatchling "
                                     "absent), so its algorithm runs as the oracle's C port"},
            "e2e": {"value": val, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _peak():
    f = ROOT / "MEASURED_PEAKS.json"
    peaks = json.loads(f.read_text()) if f.exists() else {}
    return float(peaks.get("hbm_gbs", 6650.0)), ("measured" if "hbm_gbs" in peaks else "fallback")


def _traffic(name, live_sample_steps):
    """Estimated DRAM bytes per batch of the step launches: the bytes per step
    of a warm steady-state ncu window (profiles/eng_step_<workload>_traffic.json,
    neuron + scatter launches, `window_batch` live samples) scaled by the
    batch's live sample-steps, or None without a capture."""
    base = name.removesuffix("_short")
    tf = ROOT / "profiles" / f"eng_step_{base}_traffic.json"
    if not tf.exists():
        return None
    t = json.loads(tf.read_text())
    return t["dram_bytes_per_step"] * live_sample_steps / t["window_batch"]


def job_totals(elapsed_ms: float, events: int, dev) -> tuple[float, int]:
    """Whole-job time and work of a replica run: the slowest rank's device time
    and the sum of every rank's events (one all-reduce each, every rank)."""
    import torch.distributed as dist

    return _allreduce(elapsed_ms, dev, dist.ReduceOp.MAX), int(_allreduce(events, dev, dist.ReduceOp.SUM))


def _allreduce(v, dev, op):
    import torch.distributed as dist

    t = torch.tensor([v], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=op)
    return float(t.item())


def _step_kernel(rnn):
    """What the roofline's step time covers, by the engine mode that ran."""
    mode = rnn.last_engine_choice.describe()["mode"] if rnn.last_engine_choice is not None else "?"
    if mode == "cluster":
        return ("single-cluster engine, one launch per call (state and in-edges in the shared memory of 16 SMs: "
                "HBM does not bind; profiles/cluster_engine_plain.md)")
    if mode == "tile":
        return "persistent tile engine, one launch per call"
    return f"recurrent step ({mode}: neuron + synapse launches)"


def measure(name, cfg, args, dev, world, rank, local):
    """Time args.steps whole batches of workload `name`.  Returns (line dict,
    or None on ranks > 0; model; input; lengths; network; step function; the
    last timed batch's bitmask raster)."""
    from btorch_b200.models import environ
    from btorch_b200.models.functional import reset_net

    net = make_network(cfg, args.seed)
    forced = parse_choice(args.engine_choice) if name == args.config else None
    rnn = build_model(cfg, net, dev, cfg.get("direction", args.direction))
    rnn.cudagraph = not args.no_cudagraph
    rnn.engine_status_check = "deferred"  # persistent modes: no host sync per call (checked after the timing)
    x, lens = make_inputs(cfg, args.seed + rank, dev)
    T, n = cfg["t_max"], cfg["n"]

    def one_step(xx, profile=None):
        reset_net(rnn, inplace=True)
        with torch.inference_mode(), environ.context(dt=1.0):
            raster, _ = rnn(xx, sample_len=lens, spikes_out="bitmask", engine_stats=True, engine_profile=profile,
                            engine_choice=forced)
        return raster

    for _ in range(max(3, args.warmup)):
        one_step(x)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()

    stream = torch.cuda.current_stream(dev)
    ev_start = torch.cuda.Event(enable_timing=True)
    ev_end = torch.cuda.Event(enable_timing=True)
    stats_list = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev_start.record(stream)
        last_raster = None
        for _ in range(args.steps):
            last_raster = one_step(x)
            stats_list.append(rnn.last_engine_stats.clone())
        ev_end.record(stream)
        torch.cuda.synchronize()
    elapsed_ms = ev_start.elapsed_time(ev_end)
    rnn.engine_status()  # a persistent mode's wait that gave up invalidates the timing
    launches = rnn.last_engine_launches * args.steps
    # roofline pass, outside the timed region: the same batches launched
    # eagerly with CUDA events around every projection and step launch group
    graph_mode, rnn.cudagraph = rnn.cudagraph, False
    profiles = []
    for _ in range(args.steps):
        prof = []
        one_step(x, prof)
        profiles.append(prof)
    torch.cuda.synchronize()
    rnn.cudagraph = graph_mode

    events_total = live_steps = algo_bytes = 0
    live_per_step = torch.clamp(lens.cpu()[None, :] > torch.arange(T)[:, None], 0, 1).sum(1).numpy()
    for st in stats_list:
        s = st.cpu().numpy()
        events_total += int(s[:, 1].sum())
        algo_bytes += int(8 * s[:, 2].sum() + 8 * s[:, 0].sum() + cfg["s_state"] * n * live_per_step.sum())
        live_steps += int(live_per_step.sum())
    step_ms = sum(a.elapsed_time(b) for prof in profiles for k, a, b in prof if k == "step")
    proj_ms = sum(a.elapsed_time(b) for prof in profiles for k, a, b in prof if k == "project")
    if world > 1:
        import torch.distributed as dist

        elapsed_ms, events_total = job_totals(elapsed_ms, events_total, dev)
    value = events_total / (elapsed_ms * 1e-3)
    line = None
    if rank == 0:
        peak, peak_src = _peak()
        achieved = algo_bytes / (step_ms * 1e-3) / 1e9
        traffic = _traffic(name, live_steps / args.steps)
        line = {
            "metric": "synaptic_events_per_s", "value": value, "unit": "events/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Poisson input, random weights of the configuration's shape)",
            "config": {"workload": describe(name, cfg), "direction": rnn.last_engine_direction,
                       "tuned": rnn.last_engine_choice.describe(),
                       "parallelism": f"replicas x{world}", "cudagraph": bool(rnn.cudagraph),
                       "l2": "working set (weights + input) exceeds the 126 MB L2; no flush"},
            "neuron_steps_per_s": n * live_steps / (elapsed_ms * 1e-3) if world == 1 else None,
            "spike_rate_per_step": events_total / max(1, live_steps) / len(net["w"]),
            "events_per_live_sample_step": events_total / max(1, live_steps),
            "roofline": {"bound": "hbm", "kernel": _step_kernel(rnn),
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_src, "traffic": traffic,
                         "traffic_note": "DRAM bytes per batch, scaled from profiles/eng_step_*_traffic.json",
                         "algorithmic_bytes_per_batch": algo_bytes / args.steps,
                         "step_ms_per_batch": step_ms / args.steps,
                         "projection_ms_per_batch": proj_ms / args.steps},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
    return line, rnn, x, lens, net, one_step, last_raster


def plain_step(cfg, net, x, lens, args, dev):
    """The plain single-request step: batch 1 (sample 0), eager launches."""
    from btorch_b200.models import environ
    from btorch_b200.models.functional import reset_net

    m = build_model(cfg, net, dev, args.direction, batch=1)
    m.cudagraph = False
    x1, l1 = x[:, :1].contiguous(), lens[:1]

    def go():
        reset_net(m, inplace=True)
        with torch.inference_mode(), environ.context(dt=1.0):
            return m(x1, sample_len=l1, spikes_out="bitmask", engine_stats=True)[0]

    for _ in range(2):
        go()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream(dev)
    ev = 0
    e0.record(stream)
    raster = None
    for _ in range(args.steps):
        raster = go()
        ev += m.last_engine_stats[:, 1].sum()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"value": int(ev) / (ms * 1e-3), "unit": "events/s", "ms_per_step": ms / args.steps,
            "batch": 1, "cudagraph": False, "direction": m.last_engine_direction,
            "gpu_launches": m.last_engine_launches * args.steps, "_raster": raster}


def main():
    args = parse()
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        # host cores only: rank 0 times the CPU algorithm and the other ranks
        # exit, so no process group (and no GPU) is set up
        reference_arm(args, cfg, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup(args)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from btorch_b200.models import environ
    from btorch_b200.models.functional import reset_net

    line, rnn, x, lens, net, one_step, _ = measure(args.config, cfg, args, dev, world, rank, local)
    checks = rank == 0 and world == 1 and not args.no_parity
    stream = torch.cuda.current_stream(dev)
    T, B, n = cfg["t_max"], cfg["batch"], cfg["n"]
    # e2e: host buffers through the public API -- the input in pinned host
    # memory, the model on the device: the engine streams the input to the
    # device chunk by chunk and the spike raster back to pinned host memory,
    # on a copy stream overlapped with the compute
    if not args.no_e2e:
        x_host = x.cpu().pin_memory()
        r = None
        for _ in range(3):
            # the loop below holds one result while the next call runs: warm the
            # host allocator's cache of pinned output blocks the same way
            r = one_step(x_host)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ev = 0
        d2h = 0
        for _ in range(args.steps):
            r = one_step(x_host)  # returns the raster in host memory (the previous one held meanwhile)
            ev += int(rnn.last_engine_stats[:, 1].sum())
            d2h = r.numel() * r.element_size()
        e1.record(stream)
        torch.cuda.synchronize()
        rnn.engine_status()
        e2e_ms = e0.elapsed_time(e1)
        if world > 1:
            import torch.distributed as dist

            e2e_ms, ev = job_totals(e2e_ms, ev, dev)
        if rank == 0:
            line["e2e"] = {"value": ev / (e2e_ms * 1e-3), "unit": "events/s",
                           "h2d_bytes_per_step": int(x_host.numel() * 4), "d2h_bytes_per_step": int(d2h),
                           "path": "host input and raster streamed in chunks on a copy stream"}
        del x_host, r
    if args.ncu_window is not None:
        w0 = args.ncu_window

        def hook(k0):
            if k0 == w0:
                torch.cuda.synchronize()
                torch.cuda.profiler.start()
            elif k0 == w0 + 64:
                torch.cuda.synchronize()
                torch.cuda.profiler.stop()

        reset_net(rnn, inplace=True)
        rnn.cudagraph = False
        with torch.inference_mode(), environ.context(dt=1.0):
            rnn(x, sample_len=lens, spikes_out="bitmask", engine_chunk=64, engine_chunk_hook=hook,
                engine_choice=parse_choice(args.engine_choice))
        torch.cuda.synchronize()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the port's time per live sample-step on the first S steps, applied to
        # the timed batches' events per live sample-step (the rasters are the
        # same: see the parity stage)
        S = args.cpu_sample_steps
        _, t, thr, _ = cpu_sample(cfg, net, x[:S].cpu().numpy(), S)
        eps = line["events_per_live_sample_step"]
        line["cpu_baseline"] = {"value": cpu_throughput(eps, t, S * B), "unit": "events/s", "cores": thr,
                                "kind": "port",
                                "sample": f"first {S} time steps of the {B}-sample batch timed ({t:.1f} s), "
                                          f"applied to the batch's {eps:.4g} events per live sample-step",
                                "neuron_steps_per_s": n * B * S / t}
    del rnn, one_step
    torch.cuda.empty_cache()
    parity = {}
    if checks and cfg["model"] == "alif_dense_input":
        # the start-up burst of the headline workload (dense steps included)
        parity[f"{args.config}_100"] = parity_tolerance(args.config, cfg, net, x, lens, dev, min(100, T),
                                                          args.direction)
        torch.cuda.empty_cache()
    del x, lens, net
    for extra in [e for e in args.extra.split(",") if e and e != args.config]:
        ecfg = CONFIGS[extra]
        if ecfg["model"] in ("lif_train", "serving"):
            sub = (measure_training if ecfg["model"] == "lif_train" else measure_serving)(ecfg, args, dev)
            if rank == 0:
                line[extra] = sub
            torch.cuda.empty_cache()
            continue
        sub, m, xe, le, ne, _, raster = measure(extra, ecfg, args, dev, world, rank, local)
        if rank == 0 and world == 1 and ecfg["batch"] > 1 and ecfg.get("receptors", 1) == 1:
            sub["plain_step"] = plain_step(ecfg, ne, xe, le, args, dev)
            sub["vs_plain_step"] = sub["value"] / sub["plain_step"]["value"]
            # "at identical spike rasters": the plain step's raster is sample 0's of the batched run
            one = raster_bits(sub["plain_step"].pop("_raster"), ecfg["n"])[:, 0]
            k = first_divergence(one[:, None], raster_bits(raster, ecfg["n"])[:, :1])
            sub["plain_step"]["raster_equals_batch_sample0"] = bool(k == len(one))
            sub["plain_step"]["raster_equal_steps"] = k
        if rank == 0 and world == 1 and ecfg["model"] == "lif_plain" and not args.no_cpu_baseline:
            # the reference's CPU case at full length (its spike raster is kept
            # for the comparison with the timed scatter run below)
            e, t, thr, z_port = cpu_sample(ecfg, ne, xe.cpu().numpy(), ecfg["t_max"])
            sub["cpu_baseline"] = {"value": e / t, "unit": "events/s", "cores": thr, "kind": "port",
                                   "sample": f"all {ecfg['t_max']} steps ({t:.2f} s)", "ms_per_step": 1e3 * t / ecfg["t_max"]}
            if checks:
                # the port forms W z over every synapse in the reference's order;
                # the timed run is the tuner's mode (the single-cluster engine on
                # this workload sums in that order too; the scatter would not)
                parity[f"{extra}_timed_vs_port_raster_equal_steps"] = first_divergence(
                    raster_bits(raster, ecfg["n"]), z_port)
        del raster
        del m
        torch.cuda.empty_cache()
        if checks and ecfg["model"] == "lif_plain":
            parity[f"{extra}_gather"] = parity_bitwise(extra, ecfg, ne, xe, le, dev, ecfg["t_max"], "gather",
                                                       choice="gather")
            parity[f"{extra}_cluster"] = parity_bitwise(extra, ecfg, ne, xe, le, dev, ecfg["t_max"], "gather",
                                                        choice="cluster")
            parity[f"{extra}_scatter"] = parity_tolerance(extra, ecfg, ne, xe, le, dev, ecfg["t_max"], "scatter")
        if checks and ecfg["model"] == "lif_hetero_delay":
            parity[f"{extra}_200"] = parity_bitwise(extra, ecfg, ne, xe, le, dev, min(200, ecfg["t_max"]),
                                                   args.direction)
        torch.cuda.empty_cache()
        if rank == 0:
            for k in ("metric", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline",
                      "dtype", "data"):
                sub.pop(k, None)
            line[extra] = sub
        del xe, le, ne
        torch.cuda.empty_cache()
    if checks:
        line["parity"] = parity
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
