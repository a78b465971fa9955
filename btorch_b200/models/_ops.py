"""torch.autograd.Functions over the C ABI: the sparse product, one neuron
step and one exponential-PSC step.  Each forward and backward is one or two
launches of the sm_100a kernels in btorch_b200/csrc; nothing here computes
on the CPU or falls back to torch math."""

from __future__ import annotations

import weakref
from dataclasses import dataclass

import numpy as np
import torch

from .. import _lib as L

# ----------------------------------------------------------------- layout --


@dataclass
class SparseLayout:
    """Device views of one canonical COO matrix (see include/btorch_b200.h).

    n_in = n_pre * n_bins presynaptic rows (delay-expanded), n_out = posts.
    Edge arrays of the CSR view are padded to a multiple of 4 entries (+4) so
    that 128-bit vector loads never leave the allocation."""

    n_pre: int
    n_bins: int
    n_out: int
    nnz: int
    csc_ptr: torch.Tensor   # int32 [n_out + 1]
    csc_src: torch.Tensor   # int32 (uint32 bits) [nnz]: pre | bin << 25
    csr_ptr: torch.Tensor   # int32 [n_pre + 1]
    csr_dst: torch.Tensor   # int32 (uint32 bits) [pad4(nnz)]: post | bin << 25
    csr_perm: torch.Tensor  # int64 [nnz]: CSR position -> canonical index

    @property
    def n_in(self) -> int:
        return self.n_pre * self.n_bins

    def to(self, device) -> "SparseLayout":
        return SparseLayout(self.n_pre, self.n_bins, self.n_out, self.nnz,
                            *(t.to(device) for t in (self.csc_ptr, self.csc_src, self.csr_ptr,
                                                     self.csr_dst, self.csr_perm)))


def pad4(n: int) -> int:
    return (n + 3) // 4 * 4 + 4


def build_layout(indices: torch.Tensor, n_pre: int, n_out: int, n_bins: int = 1) -> SparseLayout:
    """indices: canonical (2, nnz) int64 (post, src) with src = pre*n_bins + bin.
    Runs the host builder of the C ABI (one counting-sort pass)."""
    idx = indices.detach().to("cpu", torch.int64).contiguous()
    nnz = int(idx.shape[1])
    post = idx[0].contiguous().numpy()
    src = idx[1].contiguous().numpy()
    csc_ptr = np.zeros(n_out + 1, np.int32)
    csc_src = np.zeros(max(nnz, 1), np.uint32)
    csr_ptr = np.zeros(n_pre + 1, np.int32)
    csr_dst = np.zeros(pad4(nnz), np.uint32)
    csr_perm = np.zeros(max(nnz, 1), np.int32)
    st = L.lib().bt_layout_build(nnz, post.ctypes.data, src.ctypes.data, n_out, n_pre, n_bins,
                                 csc_ptr.ctypes.data, csc_src.ctypes.data, csr_ptr.ctypes.data,
                                 csr_dst.ctypes.data, csr_perm.ctypes.data)
    L.check(st, "bt_layout_build")
    as_t = lambda a: torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a)  # noqa: E731
    return SparseLayout(n_pre=n_pre, n_bins=n_bins, n_out=n_out, nnz=nnz, csc_ptr=as_t(csc_ptr),
                        csc_src=as_t(csc_src[:nnz].copy()), csr_ptr=as_t(csr_ptr), csr_dst=as_t(csr_dst),
                        csr_perm=torch.from_numpy(csr_perm[:nnz].astype(np.int64)))


@dataclass
class SliceLayout:
    """SELL-32 view of a layout's CSC (see bt_layout_slices)."""

    rows: int
    sl_ptr: torch.Tensor    # int64 [ceil(n/32) + 1]
    sl_src: torch.Tensor    # int32 (uint32 bits) [rows * 32]
    sl_index: torch.Tensor  # int64 [rows * 32]: canonical edge index, nnz on padding


def build_slices(layout: SparseLayout, device) -> SliceLayout:
    n = layout.n_out
    csc_ptr = layout.csc_ptr.cpu().numpy()
    csc_src = layout.csc_src.cpu().numpy().view(np.uint32)
    n_sl = (n + 31) // 32
    sl_ptr = np.zeros(n_sl + 1, np.int64)
    rows = np.zeros(1, np.int64)
    lib = L.lib()
    L.check(lib.bt_layout_slices(n, csc_ptr.ctypes.data, csc_src.ctypes.data, layout.n_pre, sl_ptr.ctypes.data,
                                 None, None, 0, rows.ctypes.data), "bt_layout_slices")
    R = int(rows[0])
    sl_src = np.zeros(max(1, R * 32), np.uint32)
    sl_perm = np.zeros(max(1, R * 32), np.int32)
    L.check(lib.bt_layout_slices(n, csc_ptr.ctypes.data, csc_src.ctypes.data, layout.n_pre, sl_ptr.ctypes.data,
                                 sl_src.ctypes.data, sl_perm.ctypes.data, R, rows.ctypes.data), "bt_layout_slices")
    idx = sl_perm.astype(np.int64)
    idx[idx < 0] = layout.nnz
    return SliceLayout(rows=R, sl_ptr=torch.from_numpy(sl_ptr).to(device),
                       sl_src=torch.from_numpy(sl_src.view(np.int32)).to(device),
                       sl_index=torch.from_numpy(idx).to(device))


def pack_slice_weights(sl: SliceLayout, w_canonical: torch.Tensor) -> torch.Tensor:
    w_ext = torch.cat([w_canonical.detach().float().reshape(-1), w_canonical.new_zeros(1, dtype=torch.float32)])
    return w_ext.index_select(0, sl.sl_index).contiguous()


def pack_csr_weights(layout: SparseLayout, w_canonical: torch.Tensor) -> torch.Tensor:
    """Weights in CSR order, padded like csr_dst (zeros in the padding)."""
    out = torch.zeros(pad4(layout.nnz), device=w_canonical.device, dtype=torch.float32)
    if layout.nnz:
        out[: layout.nnz] = w_canonical.detach().index_select(0, layout.csr_perm)
    return out


# ---------------------------------------------------------- sparse product --


def _spmv(direction: str, layout: SparseLayout, x: torch.Tensor, w_canon: torch.Tensor,
          w_csr: torch.Tensor | None) -> torch.Tensor:
    B, n_in = x.shape
    dev = x.device
    out = torch.empty((B, layout.n_out), device=dev, dtype=torch.float32)
    s = L.stream_of(dev)
    if direction == "gather":
        bits = torch.empty(max(1, B * ((n_in + 31) // 32)), device=dev, dtype=torch.int32)
        st = L.lib().bt_spmv_gather(B, n_in, layout.n_out, layout.csc_ptr.data_ptr(), layout.csc_src.data_ptr(),
                                    w_canon.data_ptr(), x.data_ptr(), out.data_ptr(), bits.data_ptr(), s)
        L.check(st, "bt_spmv_gather")
    else:
        if w_csr is None:
            w_csr = pack_csr_weights(layout, w_canon)
        work = torch.empty(B * n_in + 2, device=dev, dtype=torch.int32)
        st = L.lib().bt_spmv_scatter(B, n_in, layout.n_out, layout.csr_ptr.data_ptr(), layout.csr_dst.data_ptr(),
                                     w_csr.data_ptr(), x.data_ptr(), out.data_ptr(), work.data_ptr(), s)
        L.check(st, "bt_spmv_scatter")
    return out


class SparseMM(torch.autograd.Function):
    """out = x @ W for a SparseConn (replaces _TritonSparseMM,
    btorch/models/_sparse_triton.py:358-415)."""

    @staticmethod
    def forward(ctx, x, w_canon, layout, direction, w_csr):
        ctx.layout = layout
        ctx.save_for_backward(x, w_canon)
        ctx.w_csr = w_csr
        return _spmv(direction, layout, x, w_canon, w_csr)

    @staticmethod
    def backward(ctx, g):
        x, w_canon = ctx.saved_tensors
        layout: SparseLayout = ctx.layout
        g = g.contiguous()
        B, n_in = x.shape
        s = L.stream_of(g.device)
        gx = gw = None
        if ctx.needs_input_grad[0]:
            w_csr = ctx.w_csr if ctx.w_csr is not None else _csr_weights_cached(layout, w_canon)
            gx = torch.empty_like(x)
            gT = torch.empty(max(1, B * layout.n_out), device=g.device, dtype=torch.float32)
            L.check(L.lib().bt_spmv_grad_input_t(B, n_in, layout.n_out, layout.csr_ptr.data_ptr(),
                                                 layout.csr_dst.data_ptr(), w_csr.data_ptr(), g.data_ptr(),
                                                 gx.data_ptr(), gT.data_ptr(), s), "bt_spmv_grad_input_t")
        if ctx.needs_input_grad[1] and layout.nnz == 0:
            gw = torch.zeros(0, device=g.device, dtype=torch.float32)
        elif ctx.needs_input_grad[1]:
            gw = torch.empty(layout.nnz, device=g.device, dtype=torch.float32)
            masks = torch.empty(max(1, n_in * ((B + 31) // 32)), device=g.device, dtype=torch.int32)
            L.check(L.lib().bt_spmv_grad_weight(B, n_in, layout.n_out, layout.csc_ptr.data_ptr(),
                                                layout.csc_src.data_ptr(), x.data_ptr(), g.data_ptr(),
                                                gw.data_ptr(), masks.data_ptr(), s), "bt_spmv_grad_weight")
        return gx, gw, None, None, None


def _csr_weights_cached(layout, w):
    """Weights in CSR order for the transpose gather, packed once per weight
    tensor object and version: a SparseConn's weight is its magnitude
    parameter, the same tensor in every step of a window until the optimizer
    updates it (weak reference, so a new tensor at a reused address misses)."""
    hit = getattr(layout, "_w_csr_cache", None)
    if hit is not None and hit[0]() is w and hit[1] == (w.data_ptr(), _version(w)):
        return hit[2]
    packed = pack_csr_weights(layout, w.detach())
    layout._w_csr_cache = (weakref.ref(w), (w.data_ptr(), _version(w)), packed)
    return packed


def sparse_mm(x2d, w_canon, layout, direction, w_csr=None):
    L.require_cuda(x2d, w_canon, what="SparseConn")
    if x2d.dtype != torch.float32 or w_canon.dtype != torch.float32:
        raise TypeError("SparseConn supports float32 only.")
    x2d = x2d.contiguous()
    if torch.is_grad_enabled() and (x2d.requires_grad or w_canon.requires_grad):
        return SparseMM.apply(x2d, w_canon, layout, direction, w_csr)
    return _spmv(direction, layout, x2d, w_canon.detach(), w_csr)


# ----------------------------------------------------------- neuron step --

def exp_euler_coef(tau: torch.Tensor, dt: float, owner=None, name: str = "") -> torch.Tensor:
    """expm1(dt * lin) / lin with lin = -1.0 / tau, evaluated by torch on the
    CPU exactly as the reference's exp_euler_step does (ode.py:50), so the
    device sees the reference's fp32 value.

    With an `owner` module the result is cached on that module, keyed by dt and
    the identity and version of its `tau` tensor, so repeated steps do not copy
    the time constant back to the host."""
    key = (float(dt), tau.data_ptr(), _version(tau), tuple(tau.shape), str(tau.device))
    slot = f"_bt_coef_{name}"
    if owner is not None:
        hit = owner.__dict__.get(slot)
        if hit is not None and hit[0] == key:
            return hit[1]
    with torch.inference_mode(False):  # a normal tensor, so its version is tracked
        t_cpu = tau.detach().to("cpu", torch.float32)
        lin = -1.0 / t_cpu
        coef = (torch.expm1(dt * lin) / lin).reshape(-1).contiguous().to(tau.device)
    if owner is not None:
        owner.__dict__[slot] = (key, coef)
    return coef


def _flat(t: torch.Tensor) -> torch.Tensor:
    t = t.detach()
    if t.dtype != torch.float32:
        t = t.float()
    return t.reshape(-1).contiguous()


_SCALARS: dict = {}  # id(tensor) -> (weakref to it, (address, version), value)


def _version(t: torch.Tensor) -> int:
    # inference tensors keep no version counter (they cannot be modified
    # outside inference mode)
    return -1 if t.is_inference() else t._version


def scalar_values(tensors) -> list[float] | None:
    """Host copies of one-element tensors, or None if any has more elements.

    Cached per tensor object (by identity, never by tensor equality, which
    would synchronise) and keyed by its storage address and version counter,
    so a value is copied to the host once (one synchronisation for all
    misses) and again only after the tensor is modified in place or rebound
    to new storage."""
    if any(t.numel() != 1 for t in tensors):
        return None
    out, missing = [None] * len(tensors), []
    for i, t in enumerate(tensors):
        hit = _SCALARS.get(id(t))
        if hit is not None and hit[0]() is t and hit[1] == (t.data_ptr(), _version(t)):
            out[i] = hit[2]
        else:
            missing.append(i)
    if missing:
        vals = torch.stack([tensors[i].detach().reshape(()).to(torch.float32) for i in missing]).cpu().tolist()
        if len(_SCALARS) > 4096:  # drop entries of collected tensors
            for key in [k for k, v in _SCALARS.items() if v[0]() is None]:
                del _SCALARS[key]
        for i, v in zip(missing, vals):
            t = tensors[i]
            _SCALARS[id(t)] = (weakref.ref(t), (t.data_ptr(), _version(t)), v)
            out[i] = v
    return out


_FAST_DIV: dict = {}  # fp32 bit pattern of a divisor -> verified on the device


def fast_division(c: float, device) -> tuple[bool, float]:
    """(usable, reciprocal) for the reciprocal division of the kernels by the
    scalar divisor c: its correctly rounded reciprocal, and whether
    bt_fast_div_check found the fast quotient equal to the IEEE quotient for
    every fp32 input (checked once per divisor value and process; powers of
    two need no check, the kernels multiply by their exact reciprocal)."""
    c32 = np.float32(c)
    if not np.isfinite(c32) or c32 == 0:
        return False, 0.0
    r32 = np.float32(1.0) / c32
    mant = int(c32.view(np.uint32)) & 0x7FFFFF
    if mant == 0:
        return False, float(r32)
    key = int(c32.view(np.uint32))
    if key not in _FAST_DIV:
        m = torch.zeros(1, dtype=torch.int32, device=device)
        L.check(L.lib().bt_fast_div_check(float(c32), float(r32), m.data_ptr(), L.stream_of(device)),
                "bt_fast_div_check")
        _FAST_DIV[key] = int(m.item()) == 0
    return _FAST_DIV[key], float(r32)


_DESC_PARAMS = ("v_threshold", "v_reset", "c_m", "tau_ref", "g_leak", "E_leak", "E_k", "dg_k", "tau_adapt", "tau")


def _desc_key(node, dt):
    """What neuron_desc reads from `node`: parameter tensors by identity,
    storage and version (no values, so no synchronisation), plus the flags."""
    sg = node.surrogate_function
    key = [float(dt), type(node), bool(node.hard_reset), bool(node._use_refractory),
           getattr(sg, "spiking", True), getattr(sg, "slope", None), getattr(sg, "damping_factor", None)]
    for name in _DESC_PARAMS:
        t = getattr(node, name, None)
        key.append((id(t), t.data_ptr(), _version(t), tuple(t.shape)) if torch.is_tensor(t) else t)
    return tuple(key)


def neuron_desc(node, dt: float):
    """bt_neuron_desc for an LIF/ALIF module; returns (desc, keepalive).  When
    every parameter is a scalar, their values are also passed by value
    (desc.uniform), so the kernels read no parameter memory.

    Cached on the module until a parameter tensor is rebound, resized or
    modified in place (its version counter), or dt or a flag changes: the
    per-module path asks for it in every step's forward and backward."""
    key = _desc_key(node, dt)
    hit = node.__dict__.get("_bt_neuron_desc")
    if hit is not None and hit[0] == key:
        return hit[1], hit[2]
    d, keep = _build_neuron_desc(node, dt)
    node.__dict__["_bt_neuron_desc"] = (key, d, keep)
    return d, keep


def _build_neuron_desc(node, dt: float):
    from .neurons.alif import ALIF
    from .neurons.lif import LIF

    keep = []
    sources = {}
    nshape = tuple(node.n_neuron)

    def P(t, slot=None):
        t = torch.as_tensor(t)
        if t.numel() != 1:
            # the kernels read a scalar or one value per neuron: broadcast
            # anything narrower (a per-axis value) to the neuron shape
            try:
                t = torch.broadcast_to(t, nshape)
            except RuntimeError:
                raise NotImplementedError(
                    f"{type(node).__name__}: a parameter of shape {tuple(t.shape)} does not broadcast to the neuron "
                    f"shape {nshape} (per-sample parameters have no B200 kernel)") from None
        f = _flat(t)
        keep.append(f)
        if slot is not None:
            sources[slot] = t
        return L.param(f)

    d = L.BtNeuronDesc()
    sg = node.surrogate_function
    d.hard_reset = int(bool(node.hard_reset))
    d.use_refractory = int(bool(node._use_refractory))
    d.spiking = int(bool(getattr(sg, "spiking", True)))
    d.dt = float(dt)
    d.sg_alpha = float(getattr(sg, "slope", 2.0 * 1.7627471740390859))
    d.sg_damping = float(getattr(sg, "damping_factor", 1.0))
    d.v_threshold = P(node.v_threshold, 0)
    d.v_reset = P(node.v_reset, 1)
    d.c_m = P(node.c_m, 2)
    if node._use_refractory:
        d.tau_ref = P(node.tau_ref, 4)
    if isinstance(node, ALIF):
        d.kind = L.BT_NEURON_ALIF
        d.g_leak, d.E_leak = P(node.g_leak, 5), P(node.E_leak, 6)
        d.E_k, d.dg_k = P(node.E_k, 7), P(node.dg_k, 8)
        d.tau_adapt = P(node.tau_adapt, 9)
        d.coef_gk = P(exp_euler_coef(node.tau_adapt, dt, owner=node, name="gk"), 10)
    elif isinstance(node, LIF):
        d.kind = L.BT_NEURON_LIF
        d.tau = P(node.tau, 3)
    else:
        raise NotImplementedError(f"{type(node).__name__} has no B200 kernel")
    slots = sorted(sources)
    vals = scalar_values([sources[k] for k in slots])
    if vals is not None:
        d.uniform = 1
        for k, v in zip(slots, vals):
            d.sv[k] = v
        dev = sources[0].device
        den = float(np.float32(d.sv[0]) - np.float32(d.sv[1]))  # v_threshold - v_reset in fp32
        divisors = [(0, d.sv[2]), (1, den)]
        divisors.append((2, d.sv[3]) if d.kind == L.BT_NEURON_LIF else (3, d.sv[9]))
        if dev.type == "cuda":
            for bit, c in divisors:
                ok, r = fast_division(c, dev)
                if ok:
                    d.fast_div |= 1 << bit
                    d.rcp[bit] = r
    return d, keep


class NeuronStep(torch.autograd.Function):
    """One neuron step; backward is the hand-written surrogate gradient."""

    @staticmethod
    def forward(ctx, x, v, ref, gk, node, dt):
        d, keep = neuron_desc(node, dt)
        B, n = x.shape
        spike = torch.empty_like(x)
        v_out = torch.empty_like(v)
        ref_out = torch.empty_like(ref) if ref is not None else None
        gk_out = torch.empty_like(gk) if gk is not None else None
        u = torch.empty_like(x)
        mask = torch.empty_like(x)
        vch = torch.empty_like(x)
        st = L.lib().bt_neuron_step(d, B, n, x.data_ptr(), v.data_ptr(), L.ptr(ref), L.ptr(gk), v_out.data_ptr(),
                                    L.ptr(ref_out), L.ptr(gk_out), spike.data_ptr(), u.data_ptr(), mask.data_ptr(),
                                    vch.data_ptr(), L.stream_of(x.device))
        L.check(st, "bt_neuron_step")
        ctx.node, ctx.dt, ctx.keep = node, dt, keep
        ctx.save_for_backward(x, v, gk, u, spike, mask, vch)
        if ref_out is not None:
            ctx.mark_non_differentiable(ref_out)
        return spike, v_out, ref_out, gk_out

    @staticmethod
    def backward(ctx, g_spike, g_v, g_ref, g_gk):
        x, v, gk, u, spike, mask, vch = ctx.saved_tensors
        d, keep = neuron_desc(ctx.node, ctx.dt)
        B, n = x.shape
        g_x = torch.empty_like(x)
        g_vp = torch.empty_like(v)
        g_gkp = torch.empty_like(gk) if gk is not None else None
        cont = lambda t: None if t is None else t.contiguous()  # noqa: E731
        g_spike, g_v, g_gk = cont(g_spike), cont(g_v), cont(g_gk)
        st = L.lib().bt_neuron_step_backward(
            d, B, n, x.data_ptr(), L.ptr(g_spike), L.ptr(g_v), L.ptr(g_gk), u.data_ptr(), spike.data_ptr(),
            mask.data_ptr(), vch.data_ptr(), v.data_ptr(), L.ptr(gk), g_x.data_ptr(), g_vp.data_ptr(),
            L.ptr(g_gkp), int(bool(ctx.node.detach_reset)), L.stream_of(x.device))
        L.check(st, "bt_neuron_step_backward")
        return g_x, g_vp, None, g_gkp, None, None


def neuron_step(node, x, v, ref, gk, dt):
    """(spike, v, ref, gk) after one step, as new tensors."""
    for t in (x, v, ref, gk):
        if t is not None and t.shape != x.shape:  # the launch covers x's rows in every array
            raise RuntimeError(f"{type(node).__name__}: state of shape {tuple(t.shape)} does not match the input "
                               f"{tuple(x.shape)}; reset the network with one batch size.")
    L.require_cuda(x, v, what=type(node).__name__)
    for t in (x, v, ref, gk):
        if t is not None and t.dtype != torch.float32:
            raise TypeError(f"{type(node).__name__}: the B200 kernels support float32 state and input only.")
    need_grad = torch.is_grad_enabled() and any(t is not None and t.requires_grad for t in (x, v, gk))
    if need_grad:
        if any(p.requires_grad for p in node.parameters(recurse=False)):
            raise NotImplementedError("gradients with respect to neuron parameters are not implemented")
        return NeuronStep.apply(x.contiguous(), v.contiguous(), None if ref is None else ref.detach().contiguous(),
                                None if gk is None else gk.contiguous(), node, dt)
    d, keep = neuron_desc(node, dt)
    B, n = x.shape
    x = x.contiguous()
    # Fresh output tensors every step, like the reference's eager ops: a state
    # stack collected over steps must hold snapshots, not one aliased buffer.
    spike = torch.empty_like(x)
    v_out = torch.empty_like(v)
    ref_out = torch.empty_like(ref) if ref is not None else None
    gk_out = torch.empty_like(gk) if gk is not None else None
    st = L.lib().bt_neuron_step(d, B, n, x.data_ptr(), v.data_ptr(), L.ptr(ref), L.ptr(gk), v_out.data_ptr(),
                                L.ptr(ref_out), L.ptr(gk_out), spike.data_ptr(), None, None, None,
                                L.stream_of(x.device))
    L.check(st, "bt_neuron_step")
    return spike, v_out, ref_out, gk_out


# -------------------------------------------------------------- PSC step --


class PscStep(torch.autograd.Function):
    """psc' = psc + coef*((-psc)/tau) (+ wz).  The map is linear, so its
    backward is the same kernel applied to the incoming gradient."""

    @staticmethod
    def forward(ctx, psc, wz, coef, tau):
        out = torch.empty_like(psc)
        B = psc.shape[0]
        n = psc.shape[1]
        L.check(L.lib().bt_psc_step(B, n, L.param(coef), L.param(tau), psc.data_ptr(), L.ptr(wz), out.data_ptr(),
                                    L.stream_of(psc.device)), "bt_psc_step")
        ctx.coef, ctx.tau = coef, tau
        ctx.has_wz = wz is not None
        return out

    @staticmethod
    def backward(ctx, g):
        g = g.contiguous()
        gp = torch.empty_like(g)
        L.check(L.lib().bt_psc_step(g.shape[0], g.shape[1], L.param(ctx.coef), L.param(ctx.tau), g.data_ptr(), None,
                                    gp.data_ptr(), L.stream_of(g.device)), "bt_psc_step")
        return gp, (g if ctx.has_wz else None), None, None


def psc_step(psc, wz, coef, tau):
    L.require_cuda(psc, what="ExponentialPSC")
    if psc.dtype != torch.float32 or (wz is not None and wz.dtype != torch.float32):
        raise TypeError("ExponentialPSC: the B200 kernels support float32 only.")
    psc = psc.contiguous()
    wz = None if wz is None else wz.contiguous()
    if torch.is_grad_enabled() and (psc.requires_grad or (wz is not None and wz.requires_grad)):
        return PscStep.apply(psc, wz, coef, tau)
    out = torch.empty_like(psc)
    L.check(L.lib().bt_psc_step(psc.shape[0], psc.shape[1], L.param(coef), L.param(tau), psc.data_ptr(), L.ptr(wz),
                                out.data_ptr(), L.stream_of(psc.device)), "bt_psc_step")
    return out
