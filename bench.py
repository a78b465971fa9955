"""Benchmark of the B200 recurrent spiking step (one JSON line on rank 0).

Workload (default, --config batched): the batched-simulation configuration --
ALIF + exponential synapse (tau_syn 5 ms, adaptation tau 200 ms, dg_k 0.07),
N = 65536 neurons, fixed in-degree 500 (32.8M fp32 weights), batch 64 samples
with durations uniform in [200, 2000] steps, Poisson input from 2000 channels
at per-sample rates uniform in [2, 40] Hz through a dense fp32 input layer,
dt = 1 ms.  Synthetic, seeded inputs and random weights of that shape.  One
bench "step" simulates the whole batch (all 2000 time steps, finished samples
masked) through RecurrentNN's public forward.

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
    # name: N, in-degree, batch, c_in, T, rate range (Hz), duration range
    "batched": dict(n=65536, indeg=500, batch=64, c_in=2000, t_max=2000, rate=(2.0, 40.0), dur=(200, 2000),
                    w_scale=0.0030, in_gain=1.0),
    "small": dict(n=65536, indeg=500, batch=64, c_in=2000, t_max=64, rate=(2.0, 40.0), dur=(64, 64),
                  w_scale=0.0030, in_gain=1.0),
}
S_STATE = 36  # bytes per live neuron-sample per step: r/w v, psc, refractory, g_k (32) + input current read (4)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="batched", choices=sorted(CONFIGS))
    ap.add_argument("--direction", default="scatter", choices=["scatter", "gather", "auto"])
    ap.add_argument("--no-cudagraph", action="store_true", help="launch every chunk eagerly")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--ncu-window", type=int, default=None,
                    help="profile only time steps [S, S+64) (S a multiple of 64) of one extra batch after "
                         "the timed ones (cudaProfilerStart/Stop; use with ncu --profile-from-start off)")
    return ap.parse_args()


# ------------------------------------------------------------- workload --

def make_network(cfg, seed=0):
    """Canonical (post, src) arrays of a fixed in-degree network and ALIF params."""
    rng = np.random.default_rng(seed)
    n, k = cfg["n"], cfg["indeg"]
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
    return post, src, w, w_in


def build_model(cfg, post, src, w, w_in, device, direction):
    from btorch_b200.models import ALIF, DenseConn, ExponentialPSC, RecurrentNN, SparseConn
    from btorch_b200.models.functional import init_net_state

    n = cfg["n"]
    conn = SparseConn.from_canonical(post, src, w, (n, n), enforce_dale=False,
                                     sparse_config={"direction": direction})
    neuron = ALIF(n, v_threshold=1.0, v_reset=0.0, c_m=1.0, g_leak=0.05, E_leak=0.0, E_k=-1.0, tau_adapt=200.0,
                  dg_k=0.07, tau_ref=2.0, hard_reset=True)
    syn = ExponentialPSC(n, tau_syn=5.0, linear=conn)
    inp = DenseConn(cfg["c_in"], n, weight=torch.from_numpy(w_in))
    rnn = RecurrentNN(neuron, syn, neuron_inp_module=inp, update_state_names=()).to(device)
    init_net_state(rnn, batch_size=cfg["batch"], dtype=torch.float32, device=device)
    return rnn


def make_inputs(cfg, seed, device):
    g = torch.Generator(device=device).manual_seed(10_000 + seed)
    B, C, T = cfg["batch"], cfg["c_in"], cfg["t_max"]
    lo, hi = cfg["rate"]
    rates = lo + (hi - lo) * torch.rand(B, generator=g, device=device)
    p = (rates * 1e-3).view(1, B, 1).expand(T, B, C)
    x = torch.poisson(p.contiguous(), generator=g)
    dlo, dhi = cfg["dur"]
    lens = torch.randint(dlo, dhi + 1, (B,), generator=g, device=device)
    return x, lens


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

def cpu_sample(cfg, post, src, w, w_in, x_cpu, steps):
    """Oracle port of the reference's CPU step on the first `steps` time steps
    of the batch; returns (events, seconds, threads)."""
    from oracle import oracle as O

    n, B = cfg["n"], cfg["batch"]
    ptr = np.zeros(n + 1, np.int64)
    ptr[1:] = np.cumsum(np.bincount(post, minlength=n))
    lin = -1.0 / torch.as_tensor(200.0)
    coef_gk = float(torch.expm1(1.0 * lin) / lin)
    lin = -1.0 / torch.as_tensor(5.0)
    coef_syn = float(torch.expm1(1.0 * lin) / lin)
    spec = O.NetSpec(n=n, kind=1, hard_reset=True, use_ref=True, dt=1.0,
                     params={"v_threshold": 1.0, "v_reset": 0.0, "c_m": 1.0, "g_leak": 0.05, "E_leak": 0.0,
                             "E_k": -1.0, "dg_k": 0.07, "tau_adapt": 200.0, "coef_gk": coef_gk, "tau_ref": 2.0,
                             "psc_coef": coef_syn, "psc_tau": 5.0},
                     ptr=ptr, pre=src.astype(np.int32), delay=np.zeros(src.size, np.int32), w=w)
    threads = os.cpu_count() or 1
    st = O.init_state(spec, B)
    outdeg = np.bincount(src, minlength=n).astype(np.int64)
    t0 = time.perf_counter()
    xin = x_cpu[:steps].reshape(steps * B, -1)
    xp = O.linear(xin, w_in.T.copy()).reshape(steps, B, n)
    out = O.run(spec, st, xp, threads=threads)
    dt = time.perf_counter() - t0
    events = int((out["spikes"].astype(np.int64) * outdeg[None, None, :]).sum())
    return events, dt, threads


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
    if rank != 0:
        return
    post, src, w, w_in = make_network(cfg, args.seed)
    rng = np.random.default_rng(10_000 + args.seed)
    S = args.cpu_sample_steps
    rates = rng.uniform(*cfg["rate"], size=cfg["batch"])
    x = rng.poisson(np.broadcast_to((rates * 1e-3)[None, :, None], (S, cfg["batch"], cfg["c_in"]))).astype(np.float32)
    for _ in range(min(args.warmup, 1)):
        cpu_sample(cfg, post, src, w, w_in, x, 1)
    tot_e, tot_t, thr = 0, 0.0, 1
    for _ in range(args.steps):
        e, t, thr = cpu_sample(cfg, post, src, w, w_in, x, S)
        tot_e += e
        tot_t += t
    val = tot_e / tot_t
    sample = f"{S} time steps of the {cfg['batch']}-sample batch per step (of up to {cfg['t_max']})"
    line = {"metric": "synaptic_events_per_s", "value": val, "unit": "events/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"{args.config}: ALIF+ExpPSC N={cfg['n']} in-degree {cfg['indeg']} "
                                   f"batch {cfg['batch']} T<= {cfg['t_max']}", "parallelism": "replicas"},
            "cpu_baseline": {"value": val, "unit": "events/s", "cores": thr, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    cfg = CONFIGS[args.config]
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        reference_arm(args, cfg, world, rank)
        return
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from btorch_b200.models import environ
    from btorch_b200.models.functional import reset_net

    post, src, w, w_in = make_network(cfg, args.seed)
    rnn = build_model(cfg, post, src, w, w_in, dev, args.direction)
    rnn.cudagraph = not args.no_cudagraph
    x, lens = make_inputs(cfg, args.seed + rank, dev)
    T, B, n = cfg["t_max"], cfg["batch"], cfg["n"]
    outdeg = torch.bincount(torch.from_numpy(src), minlength=n).to(dev)

    def one_step(xx, profile=None):
        reset_net(rnn, inplace=True)
        with torch.inference_mode(), environ.context(dt=1.0):
            raster, _ = rnn(xx, sample_len=lens, spikes_out="bitmask", engine_stats=True, engine_profile=profile)
        return raster

    for _ in range(max(3, args.warmup)):
        one_step(x)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()

    stream = torch.cuda.current_stream(dev)
    profiles = []
    ev_start = torch.cuda.Event(enable_timing=True)
    ev_end = torch.cuda.Event(enable_timing=True)
    events_total = 0
    live_steps = 0
    algo_bytes = 0
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev_start.record(stream)
        stats_list = []
        for _ in range(args.steps):
            one_step(x)
            stats_list.append(rnn.last_engine_stats.clone())
        ev_end.record(stream)
        torch.cuda.synchronize()
    elapsed_ms = ev_start.elapsed_time(ev_end)
    launches = rnn.last_engine_launches * args.steps
    # roofline pass, outside the timed region: the same batch launched eagerly
    # with CUDA events around every projection and step launch group
    graph_mode, rnn.cudagraph = rnn.cudagraph, False
    for _ in range(args.steps):
        prof = []
        one_step(x, prof)
        profiles.append(prof)
    torch.cuda.synchronize()
    rnn.cudagraph = graph_mode
    for st in stats_list:
        s = st.cpu().numpy()
        events_total += int(s[:, 1].sum())
        live_per_step = torch.clamp(lens.cpu()[None, :] > torch.arange(T)[:, None], 0, 1).sum(1).numpy()
        algo_bytes += int(8 * s[:, 2].sum() + 8 * s[:, 0].sum() + S_STATE * n * live_per_step.sum())
        live_steps += int(live_per_step.sum())
    step_ms = sum(a.elapsed_time(b) for prof in profiles for k, a, b in prof if k == "step")
    proj_ms = sum(a.elapsed_time(b) for prof in profiles for k, a, b in prof if k == "project")

    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([elapsed_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
        e = torch.tensor([events_total], device=dev, dtype=torch.float64)
        dist.all_reduce(e)
        events_total = int(e.item())
    value = events_total / (elapsed_ms * 1e-3)

    line = None
    if rank == 0:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
        peak = float(peaks.get("hbm_gbs", 6650.0))
        peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
        achieved = algo_bytes / (step_ms * 1e-3) / 1e9
        traffic = None
        tf = ROOT / "profiles" / "eng_step_batched_traffic.json"
        if tf.exists():
            traffic = json.loads(tf.read_text()).get("dram_bytes_per_step")
        line = {
            "metric": "synaptic_events_per_s", "value": value, "unit": "events/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Poisson input, random weights of the configuration's shape)",
            "config": {"workload": f"{args.config}: ALIF+ExpPSC N={n} fixed in-degree {cfg['indeg']} "
                                   f"batch {B} durations {cfg['dur']} T_max {T} c_in {cfg['c_in']}",
                       "direction": rnn.last_engine_direction, "parallelism": f"replicas x{world}",
                       "cudagraph": bool(rnn.cudagraph),
                       "l2": "working set (262 MB weights + 1 GB input) exceeds the 126 MB L2; no flush"},
            "neuron_steps_per_s": n * live_steps / (elapsed_ms * 1e-3) if world == 1 else None,
            "spike_rate_per_step": None,
            "roofline": {"bound": "hbm", "kernel": "recurrent step (k_eng_neuron + k_eng_scatter)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_src, "traffic": traffic,
                         "algorithmic_bytes_per_batch": algo_bytes / args.steps,
                         "step_ms_per_batch": step_ms / args.steps, "projection_ms_per_batch": proj_ms / args.steps},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        line["spike_rate_per_step"] = events_total / max(1, live_steps) / n / cfg["indeg"]
    # e2e: host buffers through the public API (H2D of the input, D2H of the raster)
    if not args.no_e2e:
        x_host = x.cpu().pin_memory()
        raster_host = torch.empty((T, B, (n + 31) // 32), dtype=torch.int32).pin_memory()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ev_parts = []
        for _ in range(args.steps):
            xd = x_host.to(dev, non_blocking=True)
            r = one_step(xd)
            raster_host.copy_(r, non_blocking=True)
            ev_parts.append(rnn.last_engine_stats[:, 1].sum())
        e1.record(stream)
        torch.cuda.synchronize()
        ev = int(sum(int(p.item()) for p in ev_parts))
        e2e_ms = e0.elapsed_time(e1)
        if world > 1:
            import torch.distributed as dist

            t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
            e = torch.tensor([ev], device=dev, dtype=torch.float64)
            dist.all_reduce(e)
            ev = int(e.item())
        if rank == 0:
            line["e2e"] = {"value": ev / (e2e_ms * 1e-3), "unit": "events/s",
                           "h2d_bytes_per_step": int(x_host.numel() * 4),
                           "d2h_bytes_per_step": int(raster_host.numel() * 4)}
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
            rnn(x, sample_len=lens, spikes_out="bitmask", engine_chunk=64, engine_chunk_hook=hook)
        torch.cuda.synchronize()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        S = args.cpu_sample_steps
        x_cpu = x[:S].cpu().numpy()
        e, t, thr = cpu_sample(cfg, post, src, w, w_in, x_cpu, S)
        line["cpu_baseline"] = {"value": e / t, "unit": "events/s", "cores": thr, "kind": "port",
                                "sample": f"first {S} time steps of the {B}-sample batch ({t:.1f} s)"}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
