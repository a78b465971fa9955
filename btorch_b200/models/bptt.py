"""Fused surrogate-gradient BPTT for RecurrentNN calls that need gradients.

The per-module path builds one autograd node per module per step (neuron,
sparse product, synapse), so a truncated-BPTT window of T steps costs ~6 T
Python-level autograd nodes in the forward and as many backward calls.  For
the common training model -- LIF/ALIF neurons, an ExponentialPSC over a
SparseConn whose weight is its magnitude parameter, an optional DenseConn /
nn.Linear input layer -- this module runs the whole call as ONE autograd
Function: the forward steps through the same sm_100a kernels with
preallocated per-step buffers (no autograd graph), the backward walks the
steps in reverse with the hand-written backward kernels:

    forward, step t:  I_t = psc_{t-1} + P_t                  (rnn.py:524)
                      z_t, v_t, gk_t = neuron(I_t, v_{t-1}, gk_{t-1})
                      psc_t = psc_{t-1} + coef*((-psc_{t-1})/tau) + W z_t
    backward, step t: dz_t  = gZ_t + W^T dpsc_t               (bt_spmv_grad_input_t)
                      dI_t, dv_{t-1}, dgk_{t-1} = neuron'(dz_t, dv_t, dgk_t)
                      dpsc_{t-1} = dpsc_t + coef*((-dpsc_t)/tau) + dI_t   (bt_psc_step)
    weight gradient:  dW = sum over (t, b) of z_t[b, pre] dpsc_t[b, post], one
                      bt_spmv_grad_weight over all T * batch rows.

The input layer's projection P = inp(x) is computed for all steps at once
outside the Function, so its parameter and input gradients come from torch's
autograd.  Gradients equal the per-module path's up to fp32 summation order
(tests compare both with the reference's autograd within 1e-4).
"""

from __future__ import annotations

import torch
import torch.nn as nn

from .. import _lib as L
from . import environ
from ._ops import _csr_weights_cached, _spmv, neuron_desc, pack_csr_weights
from .functional import named_hidden_states
from .linear import SparseConn
from .neurons.alif import ALIF
from .neurons.lif import LIF
from .synapse import ExponentialPSC

MEMORY_FRACTION = 0.25  # largest share of free device memory the per-step buffers may take


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
    if rnn.neuron_inp_module is not None and not isinstance(rnn.neuron_inp_module, nn.Linear):
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


class _FusedBPTT(torch.autograd.Function):
    @staticmethod
    def forward(ctx, P, mag, v0, psc0, gk0, ref0, rnn, kinds):
        T, B, n = P.shape
        dev = P.device
        neuron, psc_mod, conn = rnn.neuron, rnn.synapse, rnn.synapse.linear
        dt = float(environ.get("dt"))
        d, keep = neuron_desc(neuron, dt)
        coef, tau = psc_mod.coefficients(dt)
        lay = conn.layout(dev)
        direction = conn.direction(B)
        w = mag.detach().float().contiguous()
        w_csr = pack_csr_weights(lay, w) if direction != "gather" else None
        s = L.stream_of(dev)
        new = lambda *shape: torch.empty(shape, device=dev, dtype=torch.float32)  # noqa: E731
        Z, I, U, M, VCH = new(T, B, n), new(T, B, n), new(T, B, n), new(T, B, n), new(T, B, n)
        Vs, Ps = new(T + 1, B, n), new(T + 1, B, n)
        Vs[0].copy_(v0)
        Ps[0].copy_(psc0)
        GKs = new(T + 1, B, n) if gk0 is not None else None
        if GKs is not None:
            GKs[0].copy_(gk0)
        REFs = new(T + 1, B, n) if ref0 is not None else None
        if REFs is not None:
            REFs[0].copy_(ref0)
        ptr = lambda A, t: None if A is None else A[t].data_ptr()  # noqa: E731
        for t in range(T):
            torch.add(Ps[t], P[t], out=I[t])
            L.check(L.lib().bt_neuron_step(d, B, n, I[t].data_ptr(), Vs[t].data_ptr(), ptr(REFs, t), ptr(GKs, t),
                                           Vs[t + 1].data_ptr(), ptr(REFs, t + 1), ptr(GKs, t + 1), Z[t].data_ptr(),
                                           U[t].data_ptr(), M[t].data_ptr(), VCH[t].data_ptr(), s), "bt_neuron_step")
            wz = _spmv(direction, lay, Z[t], w, w_csr)
            L.check(L.lib().bt_psc_step(B, n, L.param(coef), L.param(tau), Ps[t].data_ptr(), wz.data_ptr(),
                                        Ps[t + 1].data_ptr(), s), "bt_psc_step")
        # no reference to the module itself: the module's state will hold this
        # Function's outputs, and a cycle would keep the step buffers alive
        ctx.d, ctx.keep, ctx.coef, ctx.tau, ctx.lay = d, keep, coef, tau, lay
        ctx.detach_reset = int(bool(neuron.detach_reset))
        # saved through autograd, so they are freed after backward (unless
        # retain_graph) and Z, also returned, is checked for in-place changes
        ctx.save_for_backward(mag, Z, I, U, M, VCH, Vs, GKs)
        ctx.has_gk = GKs is not None
        ctx.set_materialize_grads(False)
        stack = lambda A, kind: A[1:].clone() if A is not None and kind in kinds else None  # noqa: E731
        last = lambda A: A[T].clone() if A is not None else None  # noqa: E731
        outs = [Z, stack(Vs, "v"), stack(Ps, "psc"), stack(GKs, "gk"), stack(REFs, "ref"),
                last(Vs), last(Ps), last(GKs), last(REFs)]
        for o in (outs[4], outs[8]):
            if o is not None:
                ctx.mark_non_differentiable(o)
        return tuple(outs)

    @staticmethod
    def backward(ctx, gZ, gV, gP, gGK, _gR, gvT, gpT, ggT, _grT):
        mag, Z, I, U, M, VCH, Vs, GKs = ctx.saved_tensors
        T, B, n = Z.shape
        dev = Z.device
        lay, d = ctx.lay, ctx.d
        s = L.stream_of(dev)
        w_csr = _csr_weights_cached(lay, mag)
        new = lambda *shape: torch.empty(shape, device=dev, dtype=torch.float32)  # noqa: E731
        G_psc, G_I = new(T, B, n), new(T, B, n)  # dL/dpsc_t (state after step t), dL/dP_t
        gz, gT_work = new(B, n), new(B * n)
        g_v = [new(B, n), new(B, n)]
        g_gk = [new(B, n), new(B, n)] if ctx.has_gk else None
        g_psc = torch.zeros((B, n), device=dev) if gpT is None else gpT.reshape(B, n).contiguous().clone()
        cur_v = None if gvT is None else gvT.reshape(B, n).contiguous()
        cur_gk = None if (ggT is None or not ctx.has_gk) else ggT.reshape(B, n).contiguous()
        detach_reset = ctx.detach_reset
        for t in reversed(range(T)):
            gp = G_psc[t]
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
            out_v = g_v[t & 1]
            out_gk = g_gk[t & 1] if g_gk is not None else None
            L.check(L.lib().bt_neuron_step_backward(
                d, B, n, I[t].data_ptr(), gz.data_ptr(), L.ptr(cur_v), L.ptr(cur_gk), U[t].data_ptr(),
                Z[t].data_ptr(), M[t].data_ptr(), VCH[t].data_ptr(), Vs[t].data_ptr(),
                GKs[t].data_ptr() if GKs is not None else None, G_I[t].data_ptr(), out_v.data_ptr(),
                L.ptr(out_gk), detach_reset, s), "bt_neuron_step_backward")
            # dpsc_{t-1} = dpsc_t + coef*((-dpsc_t)/tau) + dI_t
            nxt = torch.empty_like(g_psc)
            L.check(L.lib().bt_psc_step(B, n, L.param(ctx.coef), L.param(ctx.tau), gp.data_ptr(),
                                        G_I[t].data_ptr(), nxt.data_ptr(), s), "bt_psc_step")
            # step t - 1 reads what step t wrote and writes the other buffer of
            # each pair (one stream: the kernels run in order)
            g_psc, cur_v, cur_gk = nxt, out_v, out_gk
        g_mag = None
        if ctx.needs_input_grad[1]:
            g_mag = torch.empty(lay.nnz, device=dev, dtype=torch.float32)
            masks = torch.empty(max(1, n * ((T * B + 31) // 32)), device=dev, dtype=torch.int32)
            L.check(L.lib().bt_spmv_grad_weight(T * B, n, n, lay.csc_ptr.data_ptr(), lay.csc_src.data_ptr(),
                                                Z.data_ptr(), G_psc.data_ptr(), g_mag.data_ptr(), masks.data_ptr(),
                                                s), "bt_spmv_grad_weight")
            g_mag = g_mag.to(mag.dtype)
        return G_I, g_mag, cur_v, g_psc, cur_gk, None, None, None


def run(rnn, x: torch.Tensor, paths: dict):
    """One call through the fused BPTT, or None when its per-step buffers
    would not fit (the caller then steps module by module)."""
    neuron, syn = rnn.neuron, rnn.synapse
    n = neuron.size
    inp = rnn.neuron_inp_module
    P = inp(x) if inp is not None else x
    T = P.shape[0]
    v = neuron.v
    B = v.numel() // n
    P = torch.broadcast_to(P.reshape(T, -1, n), (T, B, n)).float().contiguous()
    free = torch.cuda.mem_get_info(P.device)[0]
    if 16 * (T + 1) * B * n * 4 > MEMORY_FRACTION * free:
        return None
    shape = v.shape
    v0 = v.reshape(B, n)
    psc0 = syn.psc.reshape(B, n)
    gk0 = neuron.g_k.reshape(B, n) if isinstance(neuron, ALIF) else None
    ref0 = neuron.refractory.reshape(B, n).detach() if neuron._use_refractory else None
    syn.linear._edge_weight()  # one weight per stored nonzero, or an error before any launch
    outs = _FusedBPTT.apply(P, syn.linear.magnitude, v0, psc0, gk0, ref0, rnn, frozenset(paths.values()))
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
    return Z.reshape(T, *shape), states


__all__ = ["match", "run"]
