"""CPU oracle for btorch's recurrent spiking step (ctypes wrapper of oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm, never by the btorch_b200 package.

The oracle restates the reference's CPU algorithm (native ``torch.sparse.mm``
backend plus the eager LIF/ALIF/ExponentialPSC/delay modules, see the header
of oracle.c for the file:line map).  It is pinned against the reference
itself through the golden fixtures in tests/golden (made by
tests/golden/make_golden.py from the reference checkout).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "oracle.c"
LIB = HERE / "_build" / "liboracle.so"

_f = C.POINTER(C.c_float)
_i64 = C.POINTER(C.c_int64)
_i32 = C.POINTER(C.c_int32)
_u8 = C.POINTER(C.c_uint8)


class _Net(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("batch", C.c_int64), ("steps", C.c_int64),
        ("kind", C.c_int32), ("hard_reset", C.c_int32), ("use_ref", C.c_int32),
        ("max_delay", C.c_int32), ("dt", C.c_float),
        ("vth", _f), ("vr", _f), ("cm", _f), ("tau", _f), ("tau_ref", _f),
        ("g_leak", _f), ("E_leak", _f), ("E_k", _f), ("dg_k", _f), ("tau_adapt", _f),
        ("coef_gk", _f), ("psc_coef", _f), ("psc_tau", _f),
        ("ptr", _i64), ("pre", _i32), ("delay", _i32), ("w", _f),
        ("x", _f), ("sample_len", _i32),
        ("v", _f), ("ref", _f), ("gk", _f), ("psc", _f), ("hist", _f),
        ("t0", C.c_int64),
        ("spikes", _u8), ("v_trace", _f), ("psc_trace", _f),
        ("threads", C.c_int32), ("n_rec", C.c_int32),
        ("row_ptr", _i64), ("row_col", _i32), ("row_w", _f), ("acc", _f),
        ("zmask", C.POINTER(C.c_uint64)),
    ]


def build(force: bool = False) -> Path:
    """Compile oracle.c (gcc, no FMA contraction) into oracle/_build."""
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(
        ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
         "-pthread", "-o", str(tmp), str(SRC), "-lm"],
        check=True,
    )
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(build()))
        _lib.orc_run.argtypes = [C.POINTER(_Net)]
        _lib.orc_run_events.argtypes = [C.POINTER(_Net)]
        _lib.orc_linear_mt.argtypes = [C.c_int64, C.c_int64, C.c_int64, _f, _f, _f, _f, C.c_int32]
        _lib.orc_linear_t.argtypes = [C.c_int64, C.c_int64, C.c_int64, _f, _f, _f, _f, C.c_int32]
        _lib.orc_spmm.argtypes = [C.c_int64, C.c_int64, C.c_int64, _i64, _i64, _f, _f, _f, C.c_int32]
        _lib.orc_linear.argtypes = [C.c_int64, C.c_int64, C.c_int64, _f, _f, _f, _f]
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def spmm(ptr, src, w, x, n_out, threads=1):
    """out = x @ W for a canonical CSC (ptr over post, src, w); x [B, n_in]."""
    x = _f32(x)
    B, n_in = x.shape
    ptr = np.ascontiguousarray(ptr, dtype=np.int64)
    src = np.ascontiguousarray(src, dtype=np.int64)
    w = _f32(w)
    out = np.zeros((B, n_out), np.float32)
    lib().orc_spmm(n_out, B, n_in, _p(ptr, _i64), _p(src, _i64), _p(w, _f), _p(x, _f), _p(out, _f), threads)
    return out


def linear(x, W, bias=None, threads=1):
    """x [rows, c_in] @ W[n, c_in]^T (+ bias), ascending-channel fmaf chain
    (rows split over `threads` host threads; the result does not depend on it)."""
    x = _f32(x)
    W = _f32(W)
    rows, c_in = x.shape
    n = W.shape[0]
    out = np.zeros((rows, n), np.float32)
    b = None if bias is None else _f32(bias)
    if lib().orc_linear_mt(rows, c_in, n, _p(x, _f), _p(W, _f), _p(b, _f), _p(out, _f), int(threads)) != 0:
        raise MemoryError("oracle projection failed")
    return out


def linear_t(x, W_t, bias=None, threads=1):
    """linear() from the transposed weight W_t [c_in, n] (DenseConn's weight
    transposed; the bench keeps it in this layout): the same chain per output,
    computed row by row as channel-ordered axpys."""
    x = _f32(x)
    W_t = _f32(W_t)
    rows, c_in = x.shape
    n = W_t.shape[1]
    out = np.empty((rows, n), np.float32)
    b = None if bias is None else _f32(bias)
    if lib().orc_linear_t(rows, c_in, n, _p(x, _f), _p(W_t, _f), _p(b, _f), _p(out, _f), int(threads)) != 0:
        raise MemoryError("oracle projection failed")
    return out


@dataclass
class NetSpec:
    """A recurrent network in the reference's terms, with parameters already
    rounded the way the reference rounds them (fp32, per neuron).

    Connectivity is the canonical post-major list of in-edges with an integer
    delay per edge (HeterSynapsePSC bin, or the uniform DelayedPSC delay).
    """

    n: int
    kind: int  # 0 LIF, 1 ALIF
    hard_reset: bool
    use_ref: bool
    dt: float
    params: dict  # name -> float32 array [n]
    ptr: np.ndarray  # int64 [n + 1]
    pre: np.ndarray  # int32 [nnz]
    delay: np.ndarray  # int32 [nnz]
    w: np.ndarray  # float32 [nnz]
    max_delay: int = 0
    n_rec: int = 1  # receptor columns per neuron: ptr, psc_coef, psc_tau span n * n_rec columns


def source_rows(spec: NetSpec):
    """The spec's edges by source row r = pre * (max_delay + 1) + delay (rows
    ascending; within a row, ascending PSC column): (row_ptr int64, row_col
    int32, row_w float32), built once per spec for the event-driven run."""
    cached = getattr(spec, "_rows", None)
    if cached is not None:
        return cached
    R = spec.max_delay + 1
    nc = spec.n * max(1, spec.n_rec)
    col = np.repeat(np.arange(nc, dtype=np.int64), np.diff(spec.ptr))
    key = spec.pre.astype(np.int64) * R + spec.delay.astype(np.int64)
    order = np.argsort(key, kind="stable")  # canonical order is by column: columns ascend within a row
    row_ptr = np.zeros(spec.n * R + 1, np.int64)
    np.cumsum(np.bincount(key, minlength=spec.n * R), out=row_ptr[1:])
    rows = (row_ptr, np.ascontiguousarray(col[order], np.int32), np.ascontiguousarray(spec.w[order], np.float32))
    spec._rows = rows
    return rows


@dataclass
class NetState:
    v: np.ndarray
    psc: np.ndarray
    ref: np.ndarray | None = None
    gk: np.ndarray | None = None
    hist: np.ndarray | None = None  # [max_delay + 1, B, n]
    t: int = 0
    extras: dict = field(default_factory=dict)


def init_state(spec: NetSpec, batch: int, v0=None, gk0=0.0) -> NetState:
    n = spec.n
    v = np.empty((batch, n), np.float32)
    v[:] = spec.params["v_reset"] if v0 is None else v0
    st = NetState(v=v, psc=np.zeros((batch, n * max(1, spec.n_rec)), np.float32))
    if spec.use_ref:
        st.ref = np.zeros((batch, n), np.float32)
    if spec.kind == 1:
        st.gk = np.full((batch, n), gk0, np.float32)
    st.hist = np.zeros((spec.max_delay + 1, batch, n), np.float32)
    return st


def run(spec: NetSpec, state: NetState, x, steps=None, sample_len=None, threads=None,
        want_v=False, want_psc=False, events=False):
    """Run the recurrent loop in place on `state`; returns dict(spikes, v, psc).

    events=False forms W z the reference's way, over every synapse each step
    (its cost is what the CPU baseline times); events=True pushes only the
    rows of neurons that spiked, in the same per-column order, which gives
    bit-identical results at a cost proportional to the spikes (parity checks
    at full network size)."""
    B, n = state.v.shape
    if x is not None:
        x = _f32(x)
        steps = x.shape[0] if steps is None else steps
        assert x.shape[1:] == (B, n)
    threads = threads or os.cpu_count() or 1
    nc = n * max(1, spec.n_rec)
    P = {k: _f32(np.broadcast_to(np.asarray(v, np.float32), (nc if k.startswith("psc_") else n,)))
         for k, v in spec.params.items()}
    need = ["v_threshold", "v_reset", "c_m", "psc_coef", "psc_tau"]
    need += ["tau"] if spec.kind == 0 else ["g_leak", "E_leak", "E_k", "dg_k", "tau_adapt", "coef_gk"]
    if spec.use_ref:
        need.append("tau_ref")
    for k in need:
        assert k in P, f"missing parameter {k}"
    spikes = np.zeros((steps, B, n), np.uint8)
    v_tr = np.zeros((steps, B, n), np.float32) if want_v else None
    p_tr = np.zeros((steps, B, nc), np.float32) if want_psc else None
    sl = None if sample_len is None else np.ascontiguousarray(sample_len, np.int32)
    net = _Net(
        n=n, batch=B, steps=steps, kind=spec.kind, hard_reset=int(spec.hard_reset),
        use_ref=int(spec.use_ref), max_delay=spec.max_delay, dt=spec.dt,
        vth=_p(P["v_threshold"], _f), vr=_p(P["v_reset"], _f), cm=_p(P["c_m"], _f),
        tau=_p(P.get("tau"), _f), tau_ref=_p(P.get("tau_ref"), _f),
        g_leak=_p(P.get("g_leak"), _f), E_leak=_p(P.get("E_leak"), _f), E_k=_p(P.get("E_k"), _f),
        dg_k=_p(P.get("dg_k"), _f), tau_adapt=_p(P.get("tau_adapt"), _f), coef_gk=_p(P.get("coef_gk"), _f),
        psc_coef=_p(P["psc_coef"], _f), psc_tau=_p(P["psc_tau"], _f),
        ptr=_p(spec.ptr, _i64), pre=_p(spec.pre, _i32), delay=_p(spec.delay, _i32), w=_p(spec.w, _f),
        x=_p(x, _f), sample_len=_p(sl, _i32),
        v=_p(state.v, _f), ref=_p(state.ref, _f), gk=_p(state.gk, _f), psc=_p(state.psc, _f),
        hist=_p(state.hist, _f), t0=state.t,
        spikes=_p(spikes, _u8), v_trace=_p(v_tr, _f), psc_trace=_p(p_tr, _f), threads=threads,
        n_rec=max(1, spec.n_rec),
    )
    acc = zmask = None
    if events:
        row_ptr, row_col, row_w = source_rows(spec)
        acc = np.zeros((B, nc), np.float32)
        # the history slots as per-neuron sample bit masks [H, n, ceil(B / 64)]
        W64 = (B + 63) // 64
        nz = np.zeros((state.hist.shape[0], n, W64 * 64), bool)
        nz[:, :, :B] = (state.hist != 0).transpose(0, 2, 1)
        zmask = np.ascontiguousarray(np.packbits(nz, axis=-1, bitorder="little")).view(np.uint64)
        net.row_ptr, net.row_col, net.row_w, net.acc = (_p(row_ptr, _i64), _p(row_col, _i32), _p(row_w, _f),
                                                        _p(acc, _f))
        net.zmask = zmask.ctypes.data_as(C.POINTER(C.c_uint64))
    keep = (x, P, spikes, v_tr, p_tr, sl, acc, zmask)  # noqa: F841 -- buffers live across the call
    if (lib().orc_run_events if events else lib().orc_run)(C.byref(net)) != 0:
        raise RuntimeError("oracle run failed")
    state.t += steps
    return {"spikes": spikes, "v": v_tr, "psc": p_tr}
