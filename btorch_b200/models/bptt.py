"""Fused surrogate-gradient BPTT for RecurrentNN calls that need gradients.

The per-module path builds one autograd node per module per step (neuron,
sparse product, synapse), so a truncated-BPTT window of T steps costs ~6 T
Python-level autograd nodes in the forward and as many backward calls.  For
the common training model -- LIF/ALIF neurons, an ExponentialPSC over a
SparseConn whose weight is its magnitude parameter, an optional DenseConn /
nn.Linear input layer -- this module runs the whole call as ONE autograd
Function: the forward steps through the sm_100a kernels with preallocated
buffers (no autograd graph), the backward walks the steps in reverse with the
hand-written backward kernels:

    forward, step t:  P_t = x_t W_in^T (+ b)                  (bt_input_project)
                      I_t = psc_{t-1} + P_t                  (rnn.py:524)
                      z_t, v_t, gk_t = neuron(I_t, v_{t-1}, gk_{t-1})
                      psc_t = psc_{t-1} + coef*((-psc_{t-1})/tau) + W z_t
    backward, step t: dz_t  = gZ_t + W^T dpsc_t               (bt_spmv_grad_input_t)
                      dI_t, dv_{t-1}, dgk_{t-1} = neuron'(dz_t, dv_t, dgk_t)
                      dpsc_{t-1} = dpsc_t + coef*((-dpsc_t)/tau) + dI_t   (bt_psc_step)
    weight gradients: dW = sum over (t, b) of z_t[b, pre] dpsc_t[b, post]
                      (bt_spmv_grad_weight, stored nonzeros only);
                      dW_in = sum over (t, b) of x_t[b]^T dI_t[b], over the
                      nonzero inputs only (bt_input_grad_weight).

Checkpointed recompute (RecurrentNN(grad_checkpoint=True), the reference's
per-chunk checkpoint, rnn.py:177-197): with chunks of C steps (chunk_size,
or unroll when chunk_size is None) the forward keeps only the spikes, the
requested state stacks and the state at every chunk start; the backward
recomputes each chunk's forward from its start state into chunk-sized
buffers (driving the synaptic recurrence with the stored spikes) and runs
that chunk's backward, accumulating the weight gradients chunk by chunk.
Memory is O(C batch n) for the step buffers instead of O(T batch n).
Without checkpointing every step's buffers are kept and nothing is
recomputed.  Gradients equal the per-module path's up to fp32 summation
order (tests compare both with the reference's autograd within 1e-4).
"""

from __future__ import annotations

import torch
import torch.nn as nn

from .. import _lib as L
from . import environ
from ._ops import _csr_weights_cached, _spmv, neuron_desc, pack_csr_weights
from .functional import named_hidden_states
from .linear import DenseConn, SparseConn
from .neurons.alif import ALIF
from .neurons.lif import LIF
from .synapse import ExponentialPSC

MEMORY_FRACTION = 0.25  # largest share of free device memory the step buffers may take


def match(rnn) -> tuple[dict | None, str]:
    """The state kinds to stack (key -> "v" / "psc" / "gk" / "ref") when the
    call can run through the fused BPTT, else (None, reason)."""
    neuron, syn = rnn.neuron, rnn.synapse
    if type(neuron) not in (LIF, ALIF) or neuron.pre_spike_v:
        return None, "neuron"
    if any(p.requires_grad for p in neuron.parameters(recurse=False)):
        return None, "neuron parameter gradients"
    if type(syn) is not ExponentialPSC or type(syn.linear) is not SparseConn or syn.linear.bias is not None:
        return None, "synapse"
    if rnn.syn_inp_module is not None:
        return None, "syn_inp_module"
    if rnn.neuron_inp_module is not None and type(rnn.neuron_inp_module) not in (nn.Linear, DenseConn):
        return None, "neuron_inp_module"
    if rnn.cpu_offload or rnn.cudagraph or rnn.save_grad_history:
        return None, "offload / graphs / grad history"
    if syn.linear.in_features != neuron.size or syn.linear.out_features != neuron.size:
        return None, "connectivity shape"
    if syn.linear.indices.shape[1] == 0:
        return None, "no synapses"
    paths = {}
    npath = next(name for name, m in rnn.named_modules() if m is neuron)
    spath = next(name for name, m in rnn.named_modules() if m is syn)
    for key in named_hidden_states(rnn, rnn.update_state_names, allow_buffer=rnn.allow_buffer):
        kind = {f"{npath}.v": "v", f"{npath}.g_k": "gk", f"{npath}.refractory": "ref", f"{spath}.psc": "psc"}.get(key)
        if kind is None:
            return None, f"state '{key}'"
        paths[key] = kind
    return paths, ""


def checkpoint_chunk(rnn, T: int) -> int:
    """Steps per recomputed chunk: the reference's checkpoint chunk (chunk_size,
    else unroll) with grad_checkpoint, else T (nothing recomputed)."""
    if not rnn.grad_checkpoint:
        return T
    if rnn.chunk_size is not None:
        return max(1, min(T, int(rnn.chunk_size)))
    return T if rnn.unroll is False else max(1, min(T, int(rnn.unroll)))


class _Steps:
    """The forward of one chunk into chunk-sized buffers (shared by the
    forward pass and the backward recomputation)."""

    def __init__(self, B, n, Cb, has_gk, has_ref, proj, c_in, dev):
        new = lambda *shape: torch.empty(shape, device=dev, dtype=torch.float32)  # noqa: E731
        self.I, self.U, self.M, self.VCH = new(Cb, B, n), new(Cb, B, n), new(Cb, B, n), new(Cb, B, n)
        self.Vs, self.Ps = new(Cb + 1, B, n), new(Cb + 1, B, n)
        self.GKs = new(Cb + 1, B, n) if has_gk else None
        self.REFs = new(Cb + 1, B, n) if has_ref else None
        self.Pc = new(Cb, B, n) if proj else None
        self.pw = torch.empty(max(1, Cb * B * (2 * c_in + 1)), device=dev, dtype=torch.int32) if proj else None
        self.zr = new(B, n)

    def load(self, v, p, gk, ref):
        self.Vs[0].copy_(v)
        self.Ps[0].copy_(p)
        if self.GKs is not None:
            self.GKs[0].copy_(gk)
        if self.REFs is not None:
            self.REFs[0].copy_(ref)

    def run(self, k, kc, xin, w_t, bias, Z, z_given, d, coef, tau, direction, lay, w, w_csr, s, stacks=None):
        """Steps 0 .. kc-1 of the chunk starting at step k.  z_given: drive the
        synaptic recurrence with the stored spikes Z[k + t] (recomputation)."""
        B, n = self.Vs.shape[1:]
        if self.Pc is not None:
            L.check(L.lib().bt_input_project(kc * B, xin.shape[-1], n, xin[k:k + kc].data_ptr(), w_t.data_ptr(),
                                             L.ptr(bias), self.Pc.data_ptr(), self.pw.data_ptr(), s),
                    "bt_input_project")
            P = self.Pc
        else:
            P = xin[k:k + kc]
        ptr = lambda A, t: None if A is None else A[t].data_ptr()  # noqa: E731
        for t in range(kc):
            torch.add(self.Ps[t], P[t], out=self.I[t])
            zt = self.zr if z_given else Z[k + t]
            L.check(L.lib().bt_neuron_step(d, B, n, self.I[t].data_ptr(), self.Vs[t].data_ptr(), ptr(self.REFs, t),
                                           ptr(self.GKs, t), self.Vs[t + 1].data_ptr(), ptr(self.REFs, t + 1),
                                           ptr(self.GKs, t + 1), zt.data_ptr(), self.U[t].data_ptr(),
                                           self.M[t].data_ptr(), self.VCH[t].data_ptr(), s), "bt_neuron_step")
            wz = _spmv(direction, lay, Z[k + t], w, w_csr)
            L.check(L.lib().bt_psc_step(B, n, L.param(coef), L.param(tau), self.Ps[t].data_ptr(), wz.data_ptr(),
                                        self.Ps[t + 1].data_ptr(), s), "bt_psc_step")
            if stacks is not None:
                for kind, A in (("v", self.Vs), ("psc", self.Ps), ("gk", self.GKs), ("ref", self.REFs)):
                    if stacks.get(kind) is not None:
                        stacks[kind][k + t].copy_(A[t + 1])

    def roll(self, kc):
        """The chunk's last state becomes the next chunk's first."""
        for A in (self.Vs, self.Ps, self.GKs, self.REFs):
            if A is not None:
                A[0].copy_(A[kc])


class _FusedBPTT(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xin, w_in, b_in, mag, v0, psc0, gk0, ref0, rnn, kinds, C):
        T, B = xin.shape[:2]
        dev = xin.device
        neuron, psc_mod, conn = rnn.neuron, rnn.synapse, rnn.synapse.linear
        n = neuron.size
        proj = w_in is not None
        c_in = int(xin.shape[-1]) if proj else 0
        dt = float(environ.get("dt"))
        d, keep = neuron_desc(neuron, dt)
        coef, tau = psc_mod.coefficients(dt)
        lay = conn.layout(dev)
        direction = conn.direction(B)
        w = mag.detach().float().contiguous()
        w_csr = pack_csr_weights(lay, w) if direction != "gather" else None
        w_t = w_in.detach().float().t().contiguous() if proj else None
        bias = b_in.detach().float().contiguous() if b_in is not None else None
        s = L.stream_of(dev)
        new = lambda *shape: torch.empty(shape, device=dev, dtype=torch.float32)  # noqa: E731
        n_ch = -(-T // C)
        ckpt = n_ch > 1
        Cb = C if ckpt else T
        st = _Steps(B, n, Cb, gk0 is not None, ref0 is not None, proj, c_in, dev)
        st.load(v0, psc0, gk0, ref0)
        Z = new(T, B, n)
        stacks = {kind: new(T, B, n) if kind in kinds else None for kind in ("v", "psc", "gk", "ref")}
        if gk0 is None:
            stacks["gk"] = None
        if ref0 is None:
            stacks["ref"] = None
        bounds = None
        if ckpt:
            bounds = {"v": new(n_ch, B, n), "psc": new(n_ch, B, n),
                      "gk": new(n_ch, B, n) if gk0 is not None else None,
                      "ref": new(n_ch, B, n) if ref0 is not None else None}
        for ci in range(n_ch):
            k = ci * C
            kc = min(C, T - k)
            if ckpt:
                for kind, A in (("v", st.Vs), ("psc", st.Ps), ("gk", st.GKs), ("ref", st.REFs)):
                    if bounds[kind] is not None:
                        bounds[kind][ci].copy_(A[0])
            st.run(k, kc, xin, w_t, bias, Z, False, d, coef, tau, direction, lay, w, w_csr, s, stacks)
            if ci + 1 < n_ch:
                st.roll(kc)
        kT = T - (n_ch - 1) * C  # steps of the last chunk
        last = lambda A: A[kT].clone() if A is not None else None  # noqa: E731
        outs = [Z, stacks["v"], stacks["psc"], stacks["gk"], stacks["ref"],
                last(st.Vs), last(st.Ps), last(st.GKs), last(st.REFs)]
        # no reference to the module itself: the module's state will hold this
        # Function's outputs, and a cycle would keep the step buffers alive
        ctx.d, ctx.keep, ctx.coef, ctx.tau, ctx.lay, ctx.direction = d, keep, coef, tau, lay, direction
        ctx.detach_reset = int(bool(neuron.detach_reset))
        ctx.C, ctx.n_ch, ctx.proj, ctx.c_in = C, n_ch, proj, c_in
        ctx.has_gk, ctx.has_ref = gk0 is not None, ref0 is not None
        ctx.bias = bias
        if ckpt:
            ctx.bounds = bounds
            ctx.steps = None  # recomputed chunk by chunk in backward
            del st
        else:
            ctx.bounds = None
            ctx.steps = st
        # saved through autograd, so they are freed after backward (unless
        # retain_graph) and Z, also returned, is checked for in-place changes
        ctx.save_for_backward(xin, w_in, mag, Z)
        ctx.set_materialize_grads(False)
        for o in (outs[4], outs[8]):
            if o is not None:
                ctx.mark_non_differentiable(o)
        return tuple(outs)

    @staticmethod
    def backward(ctx, gZ, gV, gP, gGK, _gR, gvT, gpT, ggT, _grT):
        xin, w_in, mag, Z = ctx.saved_tensors
        T, B, n = Z.shape
        dev = Z.device
        lay, d, C = ctx.lay, ctx.d, ctx.C
        s = L.stream_of(dev)
        w = mag.detach().float().contiguous()
        w_csr = _csr_weights_cached(lay, mag)
        w_fwd = pack_csr_weights(lay, w) if ctx.direction != "gather" else None
        w_t = w_in.detach().float().t().contiguous() if ctx.proj else None
        new = lambda *shape: torch.empty(shape, device=dev, dtype=torch.float32)  # noqa: E731
        st = ctx.steps
        if st is None:
            st = _Steps(B, n, C, ctx.has_gk, ctx.has_ref, ctx.proj, ctx.c_in, dev)
        Cb = st.I.shape[0]
        G_psc, G_I = new(Cb, B, n), new(Cb, B, n)  # dL/dpsc_t (state after step t), dL/dI_t of one chunk
        gz, gT_work = new(B, n), new(B * n)
        g_v = [new(B, n), new(B, n)]
        g_gk = [new(B, n), new(B, n)] if ctx.has_gk else None
        g_psc = torch.zeros((B, n), device=dev) if gpT is None else gpT.reshape(B, n).contiguous().clone()
        cur_v = None if gvT is None else gvT.reshape(B, n).contiguous()
        cur_gk = None if (ggT is None or not ctx.has_gk) else ggT.reshape(B, n).contiguous()
        detach_reset = ctx.detach_reset
        want_mag, want_x = ctx.needs_input_grad[3], ctx.needs_input_grad[0]
        want_w, want_b = ctx.proj and ctx.needs_input_grad[1], ctx.proj and ctx.needs_input_grad[2]
        g_mag = torch.empty(lay.nnz, device=dev, dtype=torch.float32) if want_mag else None
        mag_tmp = torch.empty_like(g_mag) if (want_mag and ctx.n_ch > 1) else None
        masks = torch.empty(max(1, n * ((Cb * B + 31) // 32)), device=dev, dtype=torch.int32) if want_mag else None
        g_wt = new(ctx.c_in, n) if want_w else None
        gw_work = torch.empty(max(1, ctx.c_in * (Cb * B + 1)), device=dev, dtype=torch.int32) if want_w else None
        g_b = torch.zeros(n, device=dev) if want_b else None
        g_x = torch.empty_like(xin) if want_x else None
        for ci in reversed(range(ctx.n_ch)):
            k = ci * C
            kc = min(C, T - k)
            if ctx.bounds is not None:
                bd = ctx.bounds
                st.load(bd["v"][ci], bd["psc"][ci], bd["gk"][ci] if bd["gk"] is not None else None,
                        bd["ref"][ci] if bd["ref"] is not None else None)
                st.run(k, kc, xin, w_t, ctx.bias, Z, True, d, ctx.coef, ctx.tau, ctx.direction, lay, w, w_fwd, s)
            for tl in reversed(range(kc)):
                t = k + tl
                gp = G_psc[tl]
                torch.add(g_psc, gP[t], out=gp) if gP is not None else gp.copy_(g_psc)
                if gV is not None:
                    cur_v = gV[t] if cur_v is None else cur_v + gV[t]
                if gGK is not None and ctx.has_gk:
                    cur_gk = gGK[t] if cur_gk is None else cur_gk + gGK[t]
                L.check(L.lib().bt_spmv_grad_input_t(B, n, n, lay.csr_ptr.data_ptr(), lay.csr_dst.data_ptr(),
                                                     w_csr.data_ptr(), gp.data_ptr(), gz.data_ptr(),
                                                     gT_work.data_ptr(), s), "bt_spmv_grad_input_t")
                if gZ is not None:
                    gz.add_(gZ[t])
                out_v = g_v[tl & 1]
                out_gk = g_gk[tl & 1] if g_gk is not None else None
                L.check(L.lib().bt_neuron_step_backward(
                    d, B, n, st.I[tl].data_ptr(), gz.data_ptr(), L.ptr(cur_v), L.ptr(cur_gk), st.U[tl].data_ptr(),
                    Z[t].data_ptr(), st.M[tl].data_ptr(), st.VCH[tl].data_ptr(), st.Vs[tl].data_ptr(),
                    st.GKs[tl].data_ptr() if st.GKs is not None else None, G_I[tl].data_ptr(), out_v.data_ptr(),
                    L.ptr(out_gk), detach_reset, s), "bt_neuron_step_backward")
                # dpsc_{t-1} = dpsc_t + coef*((-dpsc_t)/tau) + dI_t
                nxt = torch.empty_like(g_psc)
                L.check(L.lib().bt_psc_step(B, n, L.param(ctx.coef), L.param(ctx.tau), gp.data_ptr(),
                                            G_I[tl].data_ptr(), nxt.data_ptr(), s), "bt_psc_step")
                # step t - 1 reads what step t wrote and writes the other buffer of
                # each pair (one stream: the kernels run in order); the pair
                # parity restarts per chunk, so copy out of the pair first
                g_psc, cur_v, cur_gk = nxt, out_v, out_gk
            if cur_v is not None:
                cur_v = cur_v.clone()
            if cur_gk is not None:
                cur_gk = cur_gk.clone()
            rows = kc * B
            if want_mag:
                dst = g_mag if ci == ctx.n_ch - 1 else mag_tmp
                L.check(L.lib().bt_spmv_grad_weight(rows, n, n, lay.csc_ptr.data_ptr(), lay.csc_src.data_ptr(),
                                                    Z[k].data_ptr(), G_psc.data_ptr(), dst.data_ptr(),
                                                    masks.data_ptr(), s), "bt_spmv_grad_weight")
                if dst is mag_tmp:
                    g_mag.add_(mag_tmp)
            if want_w:
                L.check(L.lib().bt_input_grad_weight(rows, ctx.c_in, n, xin[k].data_ptr(), G_I.data_ptr(),
                                                     g_wt.data_ptr(), int(ci != ctx.n_ch - 1), gw_work.data_ptr(),
                                                     s), "bt_input_grad_weight")
            if want_b:
                g_b.add_(G_I[:kc].sum(dim=(0, 1)))
            if want_x:
                gi = G_I[:kc]
                # the input's own gradient (data rarely needs one): a plain GEMM
                g_x[k:k + kc] = (gi.reshape(rows, n) @ w_in.detach().float()).reshape(kc, B, -1) if ctx.proj else gi
        g_w = g_wt.t().contiguous().to(w_in.dtype) if want_w else None
        if g_mag is not None:
            g_mag = g_mag.to(mag.dtype)
        return g_x, g_w, g_b, g_mag, cur_v, g_psc, cur_gk, None, None, None, None


def _bytes_needed(T, B, n, C, kinds, has_gk, has_ref, proj, c_in):
    """Device bytes of the call's buffers (spikes, stacks, step buffers,
    chunk-start states, gradients of one chunk)."""
    n_ch = -(-T // C)
    Cb = C if n_ch > 1 else T
    per = T * (1 + len(kinds))  # spikes + requested stacks
    per += 4 * Cb + (2 + int(has_gk) + int(has_ref)) * (Cb + 1) + (Cb if proj else 0)  # step buffers
    per += (2 + int(has_gk) + int(has_ref)) * (n_ch if n_ch > 1 else 0)  # chunk-start states
    per += 2 * Cb  # gradients of a chunk
    return 4 * B * n * per + (4 * Cb * B * (2 * c_in + 1) if proj else 0)


def run(rnn, x: torch.Tensor, paths: dict):
    """One call through the fused BPTT, or None when its buffers would not
    fit (the caller then steps module by module)."""
    neuron, syn = rnn.neuron, rnn.synapse
    n = neuron.size
    inp = rnn.neuron_inp_module
    T = x.shape[0]
    v = neuron.v
    B = v.numel() // n
    if inp is not None:
        c_in = inp.in_features
        if x.shape[-1] != c_in:
            raise RuntimeError(f"RecurrentNN input has shape {tuple(x.shape)}; its input layer takes {c_in} channels.")
        xin = torch.broadcast_to(x.reshape(T, -1, c_in), (T, B, c_in)).float().contiguous()
        w_in, b_in = inp.weight, inp.bias
    else:
        c_in = 0
        xin = torch.broadcast_to(x.reshape(T, -1, n), (T, B, n)).float().contiguous()
        w_in = b_in = None
    C = checkpoint_chunk(rnn, T)
    kinds = frozenset(paths.values())
    free = torch.cuda.mem_get_info(x.device)[0]
    need = _bytes_needed(T, B, n, C, kinds, isinstance(neuron, ALIF), neuron._use_refractory, inp is not None, c_in)
    if need > MEMORY_FRACTION * free:
        return None
    shape = v.shape
    v0 = v.reshape(B, n)
    psc0 = syn.psc.reshape(B, n)
    gk0 = neuron.g_k.reshape(B, n) if isinstance(neuron, ALIF) else None
    ref0 = neuron.refractory.reshape(B, n).detach() if neuron._use_refractory else None
    syn.linear._edge_weight()  # one weight per stored nonzero, or an error before any launch
    outs = _FusedBPTT.apply(xin, w_in, b_in, syn.linear.magnitude, v0, psc0, gk0, ref0, rnn, kinds, C)
    Z, Vst, Pst, GKst, REFst, vT, pT, gT, rT = outs
    neuron.v = vT.reshape(shape)
    syn.psc = pT.reshape(syn.psc.shape)
    if gT is not None:
        neuron.g_k = gT.reshape(shape)
    if rT is not None:
        neuron.refractory = rT.reshape(shape)
    stacks = {"v": Vst, "psc": Pst, "gk": GKst, "ref": REFst}
    states = {key: stacks[kind].reshape(T, *shape) for key, kind in paths.items()}
    rnn.last_path = "fused-bptt"
    rnn.last_bptt = {"chunk": C, "recomputed": C < T, "bytes": need}
    return Z.reshape(T, *shape), states


__all__ = ["match", "run", "checkpoint_chunk"]
