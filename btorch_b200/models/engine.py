"""Fused multi-step engine behind RecurrentNN.multi_step_forward.

A RecurrentNN whose neuron is LIF/ALIF, whose synapse is ExponentialPSC,
DelayedPSC(ExponentialPSC) or HeterSynapsePSC(ExponentialPSC, up to
MAX_RECEPTORS receptor channels) over a SparseConn, and whose input module is
absent or a DenseConn/nn.Linear runs through ``bt_engine_run``: the whole
time loop on the device, one or two kernel launches per step
(btorch_b200/csrc/engine.cu), with the reference's outputs (spike stack and
requested state stacks) and final state.  The input may be resident in host
memory: it is then streamed through the device in chunks (_HostStreams).

Calls that need gradients run the fused BPTT (bptt.py) or the per-module
path; anything else the engine does not take runs the per-module path.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch
import torch.nn as nn

from .. import _lib as L
from . import autotune as _autotune
from . import environ
from . import _ops
from ._ops import build_slices, neuron_desc, pack_csr_weights, pack_slice_weights, scalar_values
from .functional import named_hidden_states
from .history import SpikeHistory
from .linear import BaseSparseConn
from .neurons.alif import ALIF
from .neurons.lif import LIF
from .synapse import DelayedPSC, ExponentialPSC, HeterSynapsePSC, receptor_sum

DEFAULT_CHUNK = 512
DENSE_FRACTION = 4  # scatter steps with at least n / DENSE_FRACTION spiking neurons are pulled densely
DEFAULT_GRAPH_CHUNK = 128  # steps per captured chunk (rounded to a multiple of the slot period)
CLUSTER_CHUNK = 1024  # the most steps per chunk (and launch) of the single-cluster engine
MAX_RECEPTORS = 16  # receptor channels per neuron the kernels take (bt_engine_desc.n_rec)


@dataclass
class EnginePlan:
    neuron: LIF
    psc_mod: ExponentialPSC        # module whose `psc` is the state the engine updates
    conn: BaseSparseConn
    inp: nn.Module | None
    n_bins: int                    # delay ring bins R
    uniform_delay: int             # DelayedPSC delay (0 otherwise)
    history: SpikeHistory | None
    top_syn: nn.Module             # RecurrentNN.synapse
    hetero: bool
    paths: dict                    # state key -> trace kind
    n_rec: int = 1                 # receptor channels (HeterSynapsePSC.n_receptor)


def _module_path(root: nn.Module, target: nn.Module) -> str | None:
    for name, m in root.named_modules():
        if m is target:
            return name
    return None


def match(rnn) -> tuple[EnginePlan | None, str]:
    """Return an EnginePlan for `rnn`, or (None, reason)."""
    neuron, syn = rnn.neuron, rnn.synapse
    if type(neuron) not in (LIF, ALIF):
        return None, f"neuron {type(neuron).__name__} has no fused kernel"
    if not getattr(neuron.surrogate_function, "spiking", True):
        return None, "smooth (non-spiking) surrogate forward"
    if neuron.pre_spike_v:
        return None, "pre_spike_v"
    if rnn.syn_inp_module is not None:
        return None, "syn_inp_module"
    hetero = False
    history = None
    uniform = 0
    n_bins = 1
    n_rec = 1
    if type(syn) is ExponentialPSC:
        psc_mod = syn
    elif type(syn) is DelayedPSC and type(syn.psc_module) is ExponentialPSC:
        psc_mod = syn.psc_module
        if syn.max_delay_steps > 1:
            uniform = syn.max_delay_steps
            n_bins = uniform + 1
            history = syn.history
    elif type(syn) is HeterSynapsePSC and type(syn.base_psc) is ExponentialPSC:
        if syn.n_receptor > MAX_RECEPTORS:
            return None, f"more than {MAX_RECEPTORS} receptor channels"
        psc_mod = syn.base_psc
        hetero = True
        n_rec = syn.n_receptor
        if syn.max_delay_steps > 1:
            n_bins = syn.max_delay_steps
            history = syn.history
    else:
        return None, f"synapse {type(syn).__name__} has no fused kernel"
    conn = psc_mod.linear
    if not isinstance(conn, BaseSparseConn):
        return None, "synapse linear is not a SparseConn"
    if conn.bias is not None:
        return None, "SparseConn bias"
    if conn.indices.shape[1] == 0:
        # the per-module path runs it (its products read no edge arrays then)
        return None, "the connection has no synapses"
    n = neuron.size
    if conn.out_features != n * n_rec or conn.in_features != n * (n_bins if hetero else 1):
        return None, "connectivity shape does not match the neuron count"
    if n_bins > L.BT_MAX_BINS:
        return None, "too many delay bins"
    inp = rnn.neuron_inp_module
    if inp is not None and not isinstance(inp, nn.Linear):
        return None, f"neuron_inp_module {type(inp).__name__}"
    # trace kinds for every requested state key (reference default: all memories)
    names = named_hidden_states(rnn, rnn.update_state_names, allow_buffer=rnn.allow_buffer)
    npath = _module_path(rnn, neuron)
    ppath = _module_path(rnn, psc_mod)
    spath = _module_path(rnn, syn)
    hpath = _module_path(rnn, history) if history is not None else None
    paths = {}
    for key in names:
        if key == f"{npath}.v":
            paths[key] = "v"
        elif key == f"{npath}.refractory":
            paths[key] = "ref"
        elif key == f"{npath}.g_k":
            paths[key] = "gk"
        elif key == f"{ppath}.psc" or (key == f"{spath}.psc" and n_rec == 1):
            paths[key] = "psc"
        elif key == f"{spath}.psc":
            paths[key] = "psc_sum"  # receptor sum of the base PSC trace
        elif hpath is not None and key == f"{hpath}.history":
            paths[key] = "history"
        else:
            return None, f"state '{key}' is not traced by the fused engine"
    plan = EnginePlan(neuron=neuron, psc_mod=psc_mod, conn=conn, inp=inp, n_bins=n_bins, uniform_delay=uniform,
                      history=history, top_syn=syn, hetero=hetero, paths=paths, n_rec=n_rec)
    return plan, ""


def _state2d(t: torch.Tensor, n: int) -> torch.Tensor:
    if t is None:
        raise RuntimeError("state not initialised; call init_net_state() first.")
    if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous():
        raise TypeError("the fused engine needs contiguous float32 CUDA state")
    return t.view(-1, n)


MAX_TILE_SMEM = 227 * 1024  # dynamic shared memory one CTA may opt into on sm_100


def tile_shape(n: int, batch: int, dev, tile_posts: int = 0):
    """(tile_posts, n_tiles) of the tile mode for this network and batch, or
    None when a tile's accumulators do not fit in shared memory.  By default
    one tile per SM (the fewest posts per CTA with every SM busy); a tuned
    choice may ask for larger tiles (fewer CTAs, each walking the spike lists
    once per step)."""
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    tp = int(tile_posts) or 32 * -(-(-(-n // sms)) // 32)
    tp = 32 * -(-tp // 32)
    P = -(-n // tp)
    if P > sms or batch > 256:
        return None
    if L.lib().bt_tile_smem_bytes(batch, tp, P) > MAX_TILE_SMEM:
        return None
    return tp, P


def cluster_shape(n: int, batch: int, sl_ptr, ctas: int = 0, n_bins: int = 1):
    """(tile_posts, n_ctas, tile_rows) of the single-cluster engine, or None
    when the tiles' state and in-edges do not fit one cluster's shared
    memory.  sl_ptr: the sliced in-edge view's slice -> first row offsets
    (host array; a post's in-edges are the same rows whatever the delay
    bins).  n_bins: delay bins (1..32), one bitmap copy each in shared memory.
    By default the most CTAs (up to 16) whose tiles hold at least 128 posts,
    else the most that fit."""
    import numpy as np

    sl_ptr = np.asarray(sl_ptr, dtype=np.int64)
    if batch > 256:
        return None

    def shape(cl):
        tp = 32 * -(-(-(-n // cl)) // 32)
        P = -(-n // tp)
        if P > 16:
            return None
        w = tp // 32
        # rows of each tile's slices, each slice rounded up to a multiple of 16
        slice_rows = -(-np.diff(sl_ptr) // 16) * 16
        acc = np.concatenate([[0], np.cumsum(slice_rows)])
        starts = np.minimum(np.arange(P + 1) * w, len(acc) - 1)
        rows = int(np.diff(acc[starts]).max(initial=0))
        smem = L.lib().bt_cluster_smem_bytes(n, batch, tp, rows, n_bins)
        if smem == 0 or smem > MAX_TILE_SMEM - 1024:  # (+ the static barriers)
            return None
        return tp, P, rows

    counts = [int(ctas)] if ctas else [16, 8, 4, 2, 1]
    for big_tiles in ((True, False) if not ctas else (False,)):
        for cl in counts:
            got = shape(cl)
            if got is not None and (not big_tiles or got[0] >= 128 or cl == 1):
                return got
    return None


def cluster_pack_index(lay, n: int, tp: int, P: int, rows: int, dev):
    """Where the cluster engine's packed in-edge arrays take their elements
    from: for tile t, group g, lane l, u, the flat index into the sliced view
    of row 4 g + u of the tile's slice holding (g, l), or -1 on padding
    ([P][rows / 4][32][4], int64 on `dev`); and the tiles' slice group
    offsets ([P][tp / 32 + 1] int32 on `dev`).  Built once per layout and
    shape (kept on the layout)."""
    import numpy as np

    cache = getattr(lay, "cluster_pack", None)
    if cache is None:
        cache = lay.cluster_pack = {}
    key = (tp, P, rows, str(dev))
    if key in cache:
        return cache[key]
    sl_ptr = np.asarray(lay.slices_ptr_host, dtype=np.int64)
    n_sl = len(sl_ptr) - 1
    G, NW = rows // 4, tp // 32
    idx = np.full((P, G, 32, 4), -1, np.int64)
    gptr = np.zeros((P, NW + 1), np.int32)
    g_, l_, u_ = np.meshgrid(np.arange(G), np.arange(32), np.arange(4), indexing="ij")
    for t in range(P):
        tile_n = min(tp, n - t * tp)
        acc = 0
        for w in range((tile_n + 31) // 32):
            s_ = t * NW + w
            r0, nr = int(sl_ptr[s_]), int(sl_ptr[s_ + 1] - sl_ptr[s_])
            ng = -(-nr // 16) * 4
            gptr[t, w] = acc
            row = g_[:ng] * 4 + u_[:ng]
            idx[t, acc:acc + ng] = np.where(row < nr, (r0 + row) * 32 + l_[:ng], -1)
            acc += ng
        gptr[t, (tile_n + 31) // 32:] = acc
    assert n_sl >= (n + 31) // 32
    out = (torch.from_numpy(idx.reshape(-1)).to(dev), torch.from_numpy(gptr.reshape(-1)).to(dev))
    cache[key] = out
    return out


def cluster_pack(sl, sl_w: torch.Tensor, index: torch.Tensor, n: int, n_bins: int = 1):
    """The packed weights (fp32) and ids (id XOR 31, padding n XOR 31; int16
    bits when n + 32 <= 65536, else int32; with delay bins int32 with the
    edge's bin in bits 20..24) of the cluster engine."""
    valid = index >= 0
    at = index.clamp(min=0)
    w = torch.where(valid, sl_w.reshape(-1).index_select(0, at), torch.zeros((), device=sl_w.device))
    src = sl.sl_src.reshape(-1).index_select(0, at)
    ids = (src & ((1 << L.BT_BIN_SHIFT) - 1)) ^ 31
    ids = torch.where(valid, ids, torch.full((), n ^ 31, dtype=ids.dtype, device=ids.device))
    if n_bins > 1:
        bins = torch.where(valid, (src >> L.BT_BIN_SHIFT) & 31, torch.zeros((), dtype=src.dtype, device=src.device))
        return w.contiguous(), (ids | (bins << 20)).contiguous()
    if n + 32 <= 65536:
        ids = torch.where(ids >= 32768, ids - 65536, ids).to(torch.int16)
    return w.contiguous(), ids.contiguous()


def slices_of(lay, dev):
    """The sliced in-edge view of a layout (built once, kept on the layout),
    with a host copy of its slice offsets."""
    sl = getattr(lay, "slices", None)
    if sl is None:
        sl = build_slices(lay, dev)
        lay.slices = sl
    if getattr(lay, "slices_ptr_host", None) is None:
        lay.slices_ptr_host = sl.sl_ptr.cpu().numpy()
    return sl


def tile_offsets(lay, edges: torch.Tensor, tp: int, P: int, dev) -> torch.Tensor:
    """The CSR rows split at the tile boundaries ([rows][P + 1] int32), cached
    on the layout per tile shape (they depend on the posts only)."""
    cache = lay.__dict__.setdefault("tile_offsets", {})
    off = cache.get((tp, P))
    if off is None:
        rows = lay.csr_ptr.numel() - 1
        off = torch.empty((rows, P + 1), device=dev, dtype=torch.int32)
        L.check(L.lib().bt_tile_offsets(rows, lay.csr_ptr.data_ptr(), edges.data_ptr(), tp, P, off.data_ptr(),
                                        L.stream_of(dev)), "bt_tile_offsets")
        cache[(tp, P)] = off
    return off


def graph_hist_len(n_bins: int) -> int:
    """History ring length for graph replay: 2 (R + 1), a multiple of the
    R + 1 spike-set slots of scatter mode and at least R + 2, so that the
    spike-set slot (t mod (R + 1)) and the history slot (t mod H) repeat with
    period H -- every chunk of a multiple of H steps then launches with the
    same slot arguments, which a captured graph hard-wires."""
    return 2 * (n_bins + 1)


def graph_chunk(n_bins: int, chunk: int | None = None) -> int:
    """Steps per captured chunk: `chunk` (default DEFAULT_GRAPH_CHUNK) rounded
    to a multiple of graph_hist_len(n_bins).  Calls whose length is a multiple
    of it replay graphs only (no eager remainder)."""
    H = graph_hist_len(n_bins)
    return H * max(1, round(int(chunk or DEFAULT_GRAPH_CHUNK) / H))


class _GraphEntry:
    """One captured chunk graph and the static buffers it is hard-wired to.

    Replay re-runs the recorded launches with the pointers and slot indices of
    the capture, so every tensor the chunk reads or writes lives here: the
    state (copied in from the modules before the first chunk and back out after
    the last), scratch, packed weights, the chunk's input and its outputs
    (copied out after each replay)."""

    def __init__(self):
        self.buf: dict[str, torch.Tensor] = {}
        self.graph = None
        self.sig = None
        self.captures = 0
        self.replays = 0
        # shorter last chunks of a call (T not a multiple of the chunk):
        # steps -> [graph, signature, launches, times seen]; captured the
        # second time a length comes (a one-off call stays eager)
        self.rest: dict[int, list] = {}

    def alloc(self, name, shape, dtype, dev, zero=False):
        t = self.buf.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, device=dev, dtype=dtype)
            self.buf[name] = t
            self.graph = None
            self.rest = {}
        if zero:
            t.zero_()
        return t


def graph_entries(rnn) -> dict:
    """The captured chunk graphs of `rnn`, keyed by launch configuration."""
    return rnn.__dict__.setdefault("_bt_engine_graphs", {})


def _check_input(plan: EnginePlan, x: torch.Tensor):
    """The shapes the kernels index by, checked before any device work: every
    state has the batch of v (a state reset at another batch size would be
    read past its end), and with an input layer x is [T, *batch,
    in_features] for that batch (the reference's nn.Linear raises on other
    widths; here a wider row would index past the projection weights)."""
    neuron, n = plan.neuron, plan.neuron.size
    states = [("v", neuron.v, n), ("psc", plan.psc_mod.psc, n * plan.n_rec)]
    if neuron._use_refractory:
        states.append(("refractory", neuron.refractory, n))
    if isinstance(neuron, ALIF):
        states.append(("g_k", neuron.g_k, n))
    rows = {name: t.numel() // width for name, t, width in states if torch.is_tensor(t)}
    if len(set(rows.values())) > 1:
        raise RuntimeError(f"network states disagree on the batch size {rows}; reset the network with one batch size.")
    if plan.inp is None:
        return  # [T, *batch, n] or broadcastable: reshape / broadcast_to raise otherwise
    c_in = plan.inp.in_features
    if x.ndim < 2 or x.shape[-1] != c_in:
        raise RuntimeError(f"RecurrentNN input has shape {tuple(x.shape)}; its input layer takes {c_in} channels.")
    v = plan.neuron.v
    if torch.is_tensor(v) and v.numel() and x.numel() != x.shape[0] * (v.numel() // plan.neuron.size) * c_in:
        raise RuntimeError(f"RecurrentNN input of shape {tuple(x.shape)} does not match the network state's batch "
                           f"{tuple(v.shape[:-1])}.")


def run(plan: EnginePlan, rnn, x: torch.Tensor, sample_len: torch.Tensor | None = None,
        chunk: int | None = None, spikes_out: str = "dense", stats: bool = False, profile: list | None = None,
        chunk_hook=None, choice: _autotune.EngineChoice | None = None):
    """Run T = x.shape[0] steps.  Returns (z [T, *batch, n] or bitmaps, states).

    With rnn.cudagraph the steps run in chunks of K (a multiple of the slot
    period, graph_hist_len) whose launches -- input projection, every step,
    the final PSC completion -- are captured once into a CUDA graph and
    replayed for every full chunk (the counterpart of the reference's
    CudaGraphRunner, btorch/models/cudagraph.py:101-242, with the state copied
    in once per call rather than once per chunk); a shorter last chunk runs
    eagerly on the same buffers the first time its length comes and is
    captured (and replayed from then on) the second time.

    profile: if a list, (kind, start_event, end_event) CUDA-event pairs are
    appended for every input-projection ("project") and recurrent-step
    ("step") launch group, recorded on the launching stream.
    chunk_hook: called as chunk_hook(k0) before the launches of the chunk
    that starts at step k0 (e.g. to open a profiler window).
    choice: delivery mode and tiles (default: the autotuner's cached or fresh
    choice for this problem shape, see autotune.py)."""
    _check_input(plan, x)
    check_pending_status(rnn)  # an earlier deferred status that has arrived
    launches = 0

    def _ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(torch.cuda.current_stream(dev))
        return e

    neuron, psc_mod, conn = plan.neuron, plan.psc_mod, plan.conn
    n = neuron.size
    dev = neuron.v.device
    # host-resident input: streamed to the device chunk by chunk and the
    # outputs streamed back, on a copy stream overlapped with the compute
    host_io = not x.is_cuda
    if host_io:
        L.require_cuda(neuron.v, what="RecurrentNN")
        if x.dtype != torch.float32:
            raise TypeError("RecurrentNN input must be float32 for the fused engine.")
        if not x.is_pinned():
            x = x.pin_memory()
    else:
        L.require_cuda(x, neuron.v, what="RecurrentNN")
    dt = float(environ.get("dt"))
    v_mod = _state2d(neuron.v, n)
    B = v_mod.shape[0]
    batch_shape = neuron.v.shape[:-1] if neuron.v.ndim > 1 else ()
    ref_mod = _state2d(neuron.refractory, n) if neuron._use_refractory else None
    gk_mod = _state2d(neuron.g_k, n) if isinstance(neuron, ALIF) else None
    n_rec = plan.n_rec
    nc = n * n_rec  # PSC columns (post * n_rec + receptor)
    psc_mod_t = _state2d(psc_mod.psc, nc)
    T = int(x.shape[0])
    words = (n + 31) // 32
    R = plan.n_bins
    inp = plan.inp
    c_in = int(x.shape[-1]) if inp is not None else n
    trace_kinds = sorted({"psc" if k == "psc_sum" else k for k in plan.paths.values()} - {"history"})

    if choice is None:
        choice = _autotune.choose(plan, rnn, x, sample_len, run)
    mode = choice.mode

    use_graph = bool(getattr(rnn, "cudagraph", False))
    if mode == L.BT_MODE_CLUSTER and chunk is None:
        # one launch per chunk, each loading the tiles' in-edges into shared
        # memory: longer chunks, while the chunk's input buffers stay small
        chunk = max(DEFAULT_GRAPH_CHUNK, min(CLUSTER_CHUNK, (64 << 20) // max(1, 4 * B * max(n, c_in))))
    if use_graph:
        H = graph_hist_len(R)
        K = graph_chunk(R, chunk)
        gkey = (str(dev), B, n, c_in, choice, R, H, K, spikes_out, tuple(trace_kinds), bool(stats),
                sample_len is not None, inp is not None)
        entry = graph_entries(rnn).setdefault(gkey, _GraphEntry())

        def alloc(name, shape, dtype, zero=False):
            return entry.alloc(name, shape, dtype, dev, zero)

        def static(name, t):
            """Static copy of t (the graph reads fixed addresses)."""
            if t is None:
                return None
            out = alloc(name, tuple(t.shape), t.dtype)
            out.copy_(t)
            return out
    else:
        H = R + 2
        K = int(chunk or DEFAULT_CHUNK)
        entry = None

        def alloc(name, shape, dtype, zero=False):
            return (torch.zeros if zero else torch.empty)(shape, device=dev, dtype=dtype)

        def static(name, t):
            return t

    desc = L.BtEngineDesc()
    keep = []
    nd, k1 = neuron_desc(neuron, dt)
    keep.append(k1)
    desc.neuron = nd
    coef, tau = psc_mod.coefficients(dt)
    keep += [coef, tau]
    desc.psc_coef, desc.psc_tau = L.param(coef), L.param(tau)
    pvals = scalar_values([coef, psc_mod.tau_syn])  # the module's own tensors: cached host copies
    if pvals is not None:
        desc.psc_uniform, desc.psc_coef_s, desc.psc_tau_s = 1, pvals[0], pvals[1]
        ok, r = _ops.fast_division(pvals[1], psc_mod.tau_syn.device)
        desc.psc_fast_div, desc.psc_rcp = int(ok), r
    desc.mode = mode
    lay = conn.engine_layout(R, plan.uniform_delay, dev)
    w = static("w", conn._edge_weight().detach().float().contiguous())
    keep.append(w)
    desc.n, desc.batch, desc.n_bins, desc.n_rec = n, B, R, n_rec
    desc.hist_len = H
    desc.csc_ptr, desc.csc_src, desc.csc_w = lay.csc_ptr.data_ptr(), lay.csc_src.data_ptr(), w.data_ptr()
    if mode == L.BT_MODE_SCATTER:
        lay_s = conn.scatter_layout(R, plan.uniform_delay, dev)
        w_csr = pack_csr_weights(lay_s, w)
        # one (post, weight) record per edge, interleaved
        edges = static("csr_edges", torch.stack([lay_s.csr_dst, w_csr.view(torch.int32)], 1).reshape(-1))
        keep += [w_csr, edges]
        desc.csr_ptr, desc.csr_edges = lay_s.csr_ptr.data_ptr(), edges.data_ptr()
        desc.bin_lo, desc.bin_hi = lay_s.bin_lo, lay_s.bin_hi
        desc.scatter_lanes = choice.scatter_lanes or (1 if lay_s.mean_row < 48 else 32)
        desc.neuron_spt = choice.neuron_spt or 4
        dense = choice.dense_rows if choice.dense_rows >= 0 else n // DENSE_FRACTION
        if dense > 0 and lay_s.bin_lo == lay_s.bin_hi:
            # steps where at least `dense` neurons spike are pulled over the
            # sliced in-edge view instead of scattered
            sl = getattr(lay, "slices", None)
            if sl is None:
                sl = build_slices(lay, dev)
                lay.slices = sl
            sl_w_d = static("sl_w", pack_slice_weights(sl, w))
            keep.append(sl_w_d)
            desc.sl_ptr, desc.sl_src, desc.sl_w = sl.sl_ptr.data_ptr(), sl.sl_src.data_ptr(), sl_w_d.data_ptr()
            desc.dense_rows = dense
        ring = alloc("ring", (B, nc), torch.float32)  # W z of the step (bt_engine_prime clears it)
        work = alloc("work", (L.lib().bt_engine_work_words(n, B, R),), torch.int32)
        keep += [ring, work]
        desc.ring, desc.work = ring.data_ptr(), work.data_ptr()
    tile_ws = None
    if mode == L.BT_MODE_TILE:
        lay_s = conn.scatter_layout(R, plan.uniform_delay, dev)
        w_csr = pack_csr_weights(lay_s, w)
        edges = static("csr_edges", torch.stack([lay_s.csr_dst, w_csr.view(torch.int32)], 1).reshape(-1))
        shape = tile_shape(n, B, dev, choice.tile_posts)
        if shape is None:
            raise NotImplementedError("tile mode: the tile accumulators do not fit in shared memory")
        tp, P = shape
        toff = tile_offsets(lay_s, edges, tp, P, dev)
        ring = alloc("ring", (B, nc), torch.float32, zero=True)  # W z handed to the final launch
        tile_ws = alloc("tile_work", (L.lib().bt_tile_work_words(B, tp, P),), torch.int32, zero=True)
        keep += [w_csr, edges, ring, tile_ws, toff]
        desc.csr_ptr, desc.csr_edges, desc.ring = lay_s.csr_ptr.data_ptr(), edges.data_ptr(), ring.data_ptr()
        desc.bin_lo = desc.bin_hi = 0
        desc.tile_posts, desc.n_tiles = tp, P
        desc.tile_off, desc.tile_work = toff.data_ptr(), tile_ws.data_ptr()
        desc.spin_limit = int(getattr(rnn, "engine_spin_limit", 0))
    if mode == L.BT_MODE_CLUSTER:
        sl = slices_of(lay, dev)
        shape = cluster_shape(n, B, lay.slices_ptr_host, choice.tile_posts, R)
        if shape is None:
            raise NotImplementedError("cluster mode: the network does not fit one cluster's shared memory")
        tp_c, P_c, rows_c = shape
        index, gptr = cluster_pack_index(lay, n, tp_c, P_c, rows_c, dev)
        # packed again only when the connection's parameters or buffers (its
        # effective weight's inputs) changed: in place (version) or replaced
        key = (tp_c, P_c, rows_c, R, str(dev),
               tuple((t.data_ptr(), t._version) for t in [*conn.parameters(), *conn.buffers()]))
        cached = getattr(conn, "_cluster_packed", None)
        if cached is not None and cached[0] == key:
            cl_w, cl_src = cached[1], cached[2]
        else:
            cl_w, cl_src = cluster_pack(sl, pack_slice_weights(sl, w), index, n, R)
            conn._cluster_packed = (key, cl_w, cl_src)
        cl_w, cl_src = static("cl_w", cl_w), static("cl_src", cl_src)
        tile_ws = alloc("tile_work", (32,), torch.int32, zero=True)  # word 2: status (a wait that gave up)
        keep += [cl_w, cl_src, gptr, tile_ws]
        desc.cl_w, desc.cl_src, desc.cl_gptr = cl_w.data_ptr(), cl_src.data_ptr(), gptr.data_ptr()
        desc.tile_posts, desc.n_tiles, desc.tile_rows = shape
        desc.tile_work = tile_ws.data_ptr()
        desc.spin_limit = int(getattr(rnn, "engine_spin_limit", 0))
    if mode == L.BT_MODE_PULL:
        sl = getattr(lay, "slices", None)
        if sl is None:
            sl = build_slices(lay, dev)
            lay.slices = sl
        sl_w = static("sl_w", pack_slice_weights(sl, w))
        masks = alloc("masks", (H, n + 1, L.lib().bt_mask_stride(B)), torch.int32, zero=True)
        keep += [sl_w, masks]
        desc.sl_ptr, desc.sl_src, desc.sl_w = sl.sl_ptr.data_ptr(), sl.sl_src.data_ptr(), sl_w.data_ptr()
        desc.masks = masks.data_ptr()
        desc.pull_words_per_warp = choice.pull_words
    if stats:
        outdeg = static("outdeg", (lay.csr_ptr[1:] - lay.csr_ptr[:-1]).to(torch.int32).contiguous())
        keep.append(outdeg)
        desc.outdeg = outdeg.data_ptr()
    # state: the modules' own tensors, updated in place (graph: static copies)
    v, ref, gk, psc = static("v", v_mod), static("ref", ref_mod), static("gk", gk_mod), static("psc", psc_mod_t)
    desc.v, desc.psc = v.data_ptr(), psc.data_ptr()
    desc.refractory = L.ptr(ref)
    desc.g_k = L.ptr(gk)
    hist = alloc("hist", (H, B, words), torch.int32, zero=True)
    keep.append(hist)
    desc.hist = hist.data_ptr()
    t0 = H
    s = L.stream_of(dev)
    hist_depth = plan.history.max_delay if plan.history is not None else 0
    want_hist_trace = "history" in plan.paths.values()
    if hist_depth:
        block = plan.history.recent_block(hist_depth).float().contiguous()  # [Dh, B, n], d steps ago
        if mode == L.BT_MODE_PULL:
            for d in range(hist_depth):
                L.check(L.lib().bt_float_to_masks(B, n, block[d].data_ptr(), masks[(t0 - 1 - d) % H].data_ptr(), s),
                        "bt_float_to_masks")
        else:
            bits = torch.empty((hist_depth, B, words), device=dev, dtype=torch.int32)
            L.check(L.lib().bt_float_to_bits(hist_depth * B, n, block.data_ptr(), bits.data_ptr(), s),
                    "bt_float_to_bits")
            for d in range(hist_depth):
                hist[(t0 - 1 - d) % H] = bits[d]
    desc.t0 = t0
    if mode == L.BT_MODE_SCATTER:
        # spike sets of the history steps whose arrivals are still pending
        L.check(L.lib().bt_engine_prime(C.byref(desc), s), "bt_engine_prime")
        launches += 1 if desc.bin_hi > 0 else 0

    # outputs (graph: chunk-sized static buffers, copied out after each chunk;
    # host input: pinned host tensors filled by the copy stream)
    odev = torch.device("cpu") if host_io else dev

    def out_tensor(shape, dtype, zero=False):
        if host_io:
            t = torch.empty(shape, dtype=dtype, pin_memory=True)
            return t.zero_() if zero else t
        return (torch.zeros if zero else torch.empty)(shape, device=dev, dtype=dtype)

    z = out_tensor((T, B, n), torch.float32) if spikes_out == "dense" else None
    raster = out_tensor((T, B, words), torch.int32)
    traces = {kind: out_tensor((T, B, nc if kind == "psc" else n), torch.float32) for kind in trace_kinds}
    stat_t = out_tensor((T, 4), torch.int64, zero=True) if stats else None
    if use_graph:
        out_c = {"raster": alloc("raster", (K, B, words), torch.int32)}
        if z is not None:
            out_c["z"] = alloc("z", (K, B, n), torch.float32)
        for kind in trace_kinds:
            out_c[kind] = alloc("trace_" + kind, (K, B, nc if kind == "psc" else n), torch.float32)
        if stats:
            out_c["stats"] = alloc("stats", (K, 4), torch.int64)
        out_full = {"raster": raster, "z": z, "stats": stat_t, **traces}

    # input
    if inp is not None:
        x3 = x.reshape(T, B, -1)
        w_t = static("w_t", inp.weight.detach().float().t().contiguous())
        bias = static("bias", inp.bias.detach().float().contiguous() if inp.bias is not None else None)
        keep += [w_t, bias]
    else:
        x3 = x.reshape(T, B, n) if x.numel() == T * B * n else torch.broadcast_to(x.reshape(T, -1, n), (T, B, n))
        if x3.dtype != torch.float32:
            raise TypeError("RecurrentNN input must be float32 for the fused engine.")
        x3 = x3.contiguous()
        if host_io and not x3.is_pinned():
            x3 = x3.pin_memory()
    if sample_len is not None:
        sl_full = torch.as_tensor(sample_len, device=dev, dtype=torch.int64).reshape(B)
    io = _HostStreams(dev, x3, K, T, (z, raster, stat_t, traces)) if host_io else None

    def chunk_inputs(k0, kc):
        """Device inputs of the chunk at k0: (projection input or None, step input, sample lengths)."""
        src = io.take(k0) if host_io else x3[k0:k0 + kc]  # host input: the prefetched device copy
        if use_graph:
            xin = alloc("x", (K, B, c_in), torch.float32)
            xin[:kc].copy_(src[:kc])
            xp = alloc("xp", (K, B, n), torch.float32) if inp is not None else xin
            if inp is None:
                xin = None
        elif inp is not None:
            xin = src[:kc].float().contiguous()
            xp = torch.empty((kc, B, n), device=dev, dtype=torch.float32)
        else:
            xin, xp = None, src[:kc]
        slc = None
        if sample_len is not None:
            slv = (sl_full - k0).clamp(0, kc).to(torch.int32)
            slc = alloc("sl", (B,), torch.int32) if use_graph else slv.contiguous()
            if use_graph:
                slc.copy_(slv)
        return xin, xp, slc

    def set_desc(k0, kc, xp, slc, outs):
        desc.x = xp.data_ptr()
        desc.sample_len = L.ptr(slc)
        desc.t0 = t0 + k0
        desc.n_steps = kc
        desc.raster = outs["raster"].data_ptr()
        desc.spikes = outs["z"].data_ptr() if outs.get("z") is not None else None
        desc.v_trace = outs["v"].data_ptr() if "v" in outs else None
        desc.psc_trace = outs["psc"].data_ptr() if "psc" in outs else None
        desc.ref_trace = outs["ref"].data_ptr() if "ref" in outs and ref is not None else None
        desc.gk_trace = outs["gk"].data_ptr() if "gk" in outs and gk is not None else None
        desc.stats = outs["stats"].data_ptr() if outs.get("stats") is not None else None

    def launch(k0, kc, xin, xp, slc, outs, stream):
        """Projection + steps of one chunk; outs maps output kind -> tensor whose
        row 0 is the chunk's first step.  Returns the number of kernel launches."""
        nl = 0
        if xin is not None:
            pw = alloc("pw", (K * B * (2 * c_in + 1),), torch.int32) if use_graph else \
                torch.empty(kc * B * (2 * c_in + 1), device=dev, dtype=torch.int32)
            keep.append(pw)
            e0 = _ev() if profile is not None else None
            if slc is not None:  # finished samples' steps are not projected
                L.check(L.lib().bt_input_project_live(kc, B, c_in, n, xin.data_ptr(), w_t.data_ptr(), L.ptr(bias),
                                                      slc.data_ptr(), xp.data_ptr(), pw.data_ptr(), stream),
                        "bt_input_project_live")
            else:
                L.check(L.lib().bt_input_project(kc * B, c_in, n, xin.data_ptr(), w_t.data_ptr(), L.ptr(bias),
                                                 xp.data_ptr(), pw.data_ptr(), stream), "bt_input_project")
            nl += 2
            if profile is not None:
                profile.append(("project", e0, _ev()))
        set_desc(k0, kc, xp, slc, outs)
        e0 = _ev() if profile is not None else None
        L.check(L.lib().bt_engine_run(C.byref(desc), stream), "bt_engine_run")
        nl += 1 if mode == L.BT_MODE_CLUSTER else 2 if mode == L.BT_MODE_TILE else \
            (2 * kc if mode == L.BT_MODE_SCATTER else kc) + 1
        if profile is not None:
            profile.append(("step", e0, _ev()))
        return nl

    if host_io:
        io.prefetch(0)
    for k0 in range(0, T, K):
        kc = min(K, T - k0)
        if chunk_hook is not None:
            chunk_hook(k0)
        if host_io and k0 + K < T:
            io.prefetch(k0 + K)
        xin, xp, slc = chunk_inputs(k0, kc)
        if not use_graph:
            if host_io:
                outs = io.device_outs(k0)
            else:
                outs = {"raster": raster[k0], "z": z[k0] if z is not None else None,
                        "stats": stat_t[k0] if stat_t is not None else None,
                        **{kind: traces[kind][k0] for kind in trace_kinds}}
            launches += launch(k0, kc, xin, xp, slc, outs, s)
            if host_io:
                io.consumed(k0)
                io.drain(k0, kc)
            continue
        if "stats" in out_c:
            out_c["stats"].zero_()
        if kc == K and profile is None:
            # every full chunk starts at the same slot phase (K is a multiple of H):
            # the capture records the launches of a chunk at k0 = 0
            set_desc(0, K, xp, slc, out_c)
            sig = _graph_signature(desc, xin, xp, slc, out_c, w_t if inp is not None else None,
                                   bias if inp is not None else None)
            if entry.graph is None or entry.sig != sig:
                # first full chunk of this configuration: run it eagerly (which
                # also performs any first-launch setup outside the capture),
                # then record the same launches for the following chunks
                nl = launch(k0, kc, xin, xp, slc, out_c, s)
                torch.cuda.synchronize(dev)
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    if "stats" in out_c:
                        out_c["stats"].zero_()
                    entry.nodes = launch(0, K, xin, xp, slc, out_c, L.stream_of(dev))
                entry.graph, entry.sig = g, sig
                entry.captures += 1
            else:
                entry.graph.replay()
                entry.replays += 1
                nl = entry.nodes
            launches += nl
        elif profile is None:
            # the call's shorter last chunk (it starts at a multiple of K: the
            # slot phase of k0 = 0, like the full chunks)
            set_desc(0, kc, xp, slc, out_c)
            sig = _graph_signature(desc, xin, xp, slc, out_c, w_t if inp is not None else None,
                                   bias if inp is not None else None)
            rest = entry.rest.setdefault(kc, [None, None, 0, 0])
            rest[3] += 1
            if rest[0] is not None and rest[1] == sig:
                rest[0].replay()
                launches += rest[2]
            else:
                launches += launch(k0, kc, xin, xp, slc, out_c, s)
                if rest[3] >= 2:
                    torch.cuda.synchronize(dev)
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g):
                        if "stats" in out_c:
                            out_c["stats"].zero_()
                        rest[2] = launch(0, kc, xin, xp, slc, out_c, L.stream_of(dev))
                    rest[0], rest[1] = g, sig
        else:
            launches += launch(k0, kc, xin, xp, slc, out_c, s)
        if host_io:
            io.consumed(k0)
            dev_outs = io.device_outs(k0)
            for kind, t in out_c.items():
                if dev_outs.get(kind) is not None:
                    dev_outs[kind][:kc].copy_(t[:kc])
            io.drain(k0, kc)
            continue
        for kind, t in out_c.items():
            if out_full.get(kind) is not None:
                out_full[kind][k0:k0 + kc].copy_(t[:kc])
    if host_io:
        io.finish()
    if tile_ws is not None:
        # the launches' status word (a wait that gave up)
        what = "tile mode: a grid barrier" if mode == L.BT_MODE_TILE else "cluster mode: a spike-word"
        if getattr(rnn, "engine_status_check", "sync") == "deferred":
            host = torch.empty(1, dtype=torch.int32, pin_memory=True)
            host.copy_(tile_ws[2:3], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(torch.cuda.current_stream(dev))
            rnn._engine_pending_status = (host, ev, what)
        else:
            status = int(tile_ws[2].item())
            if status:
                tile_ws[:32].zero_()
                raise RuntimeError(f"fused engine, {what} wait gave up (BT_ERR_TIMEOUT); "
                                   "the call's results are invalid")

    if use_graph:
        v_mod.copy_(v)
        psc_mod_t.copy_(psc)
        if ref_mod is not None:
            ref_mod.copy_(ref)
        if gk_mod is not None:
            gk_mod.copy_(gk)

    # write the spike history back into the module (last Dh spikes)
    t_end = t0 + T
    if hist_depth:
        block = torch.empty((hist_depth, B, n), device=dev, dtype=torch.float32)
        if mode == L.BT_MODE_PULL:
            for d in range(hist_depth):
                L.check(L.lib().bt_masks_to_float(B, n, masks[(t_end - 1 - d) % H].data_ptr(), block[d].data_ptr(), s),
                        "bt_masks_to_float")
        else:
            sel = torch.stack([hist[(t_end - 1 - d) % H] for d in range(hist_depth)]).contiguous()
            L.check(L.lib().bt_bits_to_float(hist_depth * B, n, sel.data_ptr(), block.data_ptr(), s),
                    "bt_bits_to_float")
        init_block = plan.history.recent_block(hist_depth).clone() if want_hist_trace else None
        plan.history.store_recent_block(block, T)
    if plan.hetero:
        lead = psc_mod.psc.shape[:-1]
        if n_rec == 1:
            plan.top_syn.psc = psc_mod.psc.view(*lead, *plan.top_syn.n_neuron)
        else:
            ps = receptor_sum(psc_mod.psc.view(*lead, n, n_rec)).view(*lead, *plan.top_syn.n_neuron)
            cur = plan.top_syn.psc
            if torch.is_tensor(cur) and cur.shape == ps.shape and cur.dtype == ps.dtype and cur.device == ps.device \
                    and not cur.is_inference():
                cur.copy_(ps)  # keep the module's own (non-inference) tensor: in-place resets stay legal
            else:
                plan.top_syn.psc = ps
    if "ref" in traces and ref is None:
        traces.pop("ref")

    states = {}
    for key, kind in plan.paths.items():
        if kind == "history":
            zz = z.to(dev) if z is not None else _expand(raster.to(dev), n)
            states[key] = _history_trace(plan.history, zz, init_block, batch_shape, None).to(odev)
        elif kind == "psc_sum":
            states[key] = receptor_sum(traces["psc"].view(T, B, n, n_rec)).view(T, *batch_shape, *plan.neuron.n_neuron)
        else:
            states[key] = traces[kind].view(T, *batch_shape, *_nshape(plan, key))
    rnn.last_engine_stats = stat_t
    rnn.last_engine_direction = {L.BT_MODE_SCATTER: "scatter", L.BT_MODE_GATHER: "gather",
                                 L.BT_MODE_PULL: "pull", L.BT_MODE_TILE: "scatter",
                                 L.BT_MODE_CLUSTER: "gather"}[mode]
    rnn.last_engine_launches = launches
    rnn.last_engine_choice = choice
    if z is not None:
        z = z.view(T, *batch_shape, *neuron.n_neuron)
        return z, states
    return raster, states


_COPY_STREAMS: dict = {}


class _HostStreams:
    """Chunked host <-> device streaming of one call with host-resident input.

    Input chunk c (steps k0 .. k0 + K) goes host -> device on a copy stream
    into one of two device staging buffers while the previous chunk computes;
    the compute stream waits for it (take) and frees the buffer once the
    chunk's launches are enqueued (consumed).  Each chunk's outputs land in one
    of two chunk-sized device buffers and go device -> host on the copy stream
    (drain), the compute stream waiting before it reuses a buffer.  Device
    memory is two chunks' worth whatever T."""

    def __init__(self, dev, x3, K, T, outs):
        self.dev, self.x3, self.K, self.T = dev, x3, K, T
        z, raster, stat_t, traces = outs
        self.host = {"raster": raster, "z": z, "stats": stat_t, **traces}
        self.cs = _COPY_STREAMS.get(dev)
        if self.cs is None:
            self.cs = _COPY_STREAMS[dev] = torch.cuda.Stream(dev)
        shape = (K,) + tuple(x3.shape[1:])
        self.stg = [torch.empty(shape, device=dev, dtype=x3.dtype) for _ in range(2)]
        self.dout = [{k: torch.empty((K,) + tuple(h.shape[1:]), device=dev, dtype=h.dtype)
                      for k, h in self.host.items() if h is not None} for _ in range(2)]
        self.ev_in, self.ev_free, self.ev_out_free = [None, None], [None, None], [None, None]

    def _par(self, k0):
        return (k0 // self.K) & 1

    def prefetch(self, k0):
        p = self._par(k0)
        kc = min(self.K, self.T - k0)
        with torch.cuda.stream(self.cs):
            if self.ev_free[p] is not None:
                self.cs.wait_event(self.ev_free[p])
            self.stg[p][:kc].copy_(self.x3[k0:k0 + kc], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.cs)
            self.ev_in[p] = ev

    def take(self, k0):
        p = self._par(k0)
        torch.cuda.current_stream(self.dev).wait_event(self.ev_in[p])
        return self.stg[p]

    def consumed(self, k0):
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.dev))
        self.ev_free[self._par(k0)] = ev

    def device_outs(self, k0):
        p = self._par(k0)
        if self.ev_out_free[p] is not None:
            torch.cuda.current_stream(self.dev).wait_event(self.ev_out_free[p])
        return self.dout[p]

    def drain(self, k0, kc):
        p = self._par(k0)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(self.cs):
            self.cs.wait_event(ev)
            for k, d in self.dout[p].items():
                self.host[k][k0:k0 + kc].copy_(d[:kc], non_blocking=True)
            done = torch.cuda.Event()
            done.record(self.cs)
        self.ev_out_free[p] = done

    def finish(self):
        self.cs.synchronize()  # host outputs complete; staging buffers idle


def check_pending_status(rnn, wait: bool = False) -> None:
    """Raise for a deferred status word of an earlier call that reports a
    wait that gave up.  Without `wait`, a status still in flight stays
    pending."""
    pend = getattr(rnn, "_engine_pending_status", None)
    if pend is None:
        return
    host, ev, what = pend
    if not wait and not ev.query():
        return
    ev.synchronize()
    rnn._engine_pending_status = None
    if int(host[0]):
        raise RuntimeError(f"fused engine, {what} wait gave up (BT_ERR_TIMEOUT) in an earlier call; "
                           "its results are invalid")


def _graph_signature(desc, *tensors):
    """Everything a captured chunk hard-wires: the descriptor's bytes (pointers,
    sizes, scalars) and the addresses of the projection's operands."""
    ptrs = []
    for t in tensors:
        if isinstance(t, dict):
            ptrs += [(k, v.data_ptr()) for k, v in sorted(t.items())]
        else:
            ptrs.append(t.data_ptr() if t is not None else 0)
    return bytes(desc), tuple(ptrs)


def _nshape(plan: EnginePlan, key: str):
    if plan.hetero and key.endswith("base_psc.psc"):
        return (plan.neuron.size * plan.n_rec,)
    return plan.neuron.n_neuron


def _expand(raster: torch.Tensor, n: int) -> torch.Tensor:
    T, B, W = raster.shape
    out = torch.empty((T, B, n), device=raster.device, dtype=torch.float32)
    L.check(L.lib().bt_bits_to_float(T * B, n, raster.data_ptr(), out.data_ptr(), L.stream_of(raster.device)),
            "bt_bits_to_float")
    return out


def _history_trace(hist_mod: SpikeHistory, z: torch.Tensor, init_block: torch.Tensor, batch_shape,
                   c0: torch.Tensor | None) -> torch.Tensor:
    """Stack of the history memory after every step, as the reference returns it.

    cat mode (history.py:233-250) rebinds a new tensor every step, so the
    stack holds true snapshots (index d = d steps ago).  Circular mode
    (history.py:218-231) writes into the same storage every step, so every
    entry of the reference's stack aliases that storage and reads as the final
    buffer; the engine returns the same."""
    T, B, n = z.shape[0], z.shape[1], z.shape[-1]
    D = hist_mod.max_delay
    if hist_mod.use_circular_buffer:
        final = hist_mod.history.reshape(*batch_shape, D, n)
        return final.unsqueeze(0).expand(T, *final.shape).clone()
    z = z.reshape(T, B, n)
    seq = torch.cat([init_block.flip(0).reshape(D, B, n), z], dim=0)  # seq[i] = z_{i - D}
    idx = torch.arange(T, device=z.device)[:, None] + D - torch.arange(D, device=z.device)[None, :]
    out = seq[idx]  # [T, D, B, n], d steps ago
    return out.permute(0, 2, 1, 3).reshape(T, *batch_shape, D, n)
