"""Generate golden vectors from the reference btorch (run in the build container).

The reference checkout is imported read-only from the directory given by
--ref, or else by the BTORCH_REFERENCE environment variable.  Each case
builds the reference's own modules on seeded
synthetic inputs, runs them on the CPU (native sparse backend, fp32) and
saves inputs, parameters and outputs to tests/golden/<case>.npz.  The tests
replay these cases through the CPU oracle (pinning it to the reference) and
through the CUDA engine.

    BTORCH_REFERENCE=<reference checkout> python tests/golden/make_golden.py
    python tests/golden/make_golden.py --ref <reference checkout>
"""

from __future__ import annotations

import argparse
import importlib.metadata as md
import os
import sys
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def _import_reference(ref_root: str):
    orig = md.version
    md.version = lambda name: "0.0.0+ref" if name == "btorch" else orig(name)
    sys.path.insert(0, ref_root)
    import torch  # noqa: F401

    import btorch  # noqa: F401
    return


def make_conn(rng, n_pre, n_post, p, dyadic, exc_frac=0.8, scale=0.1, inh_gain=-0.4, dy_exp=-8):
    """(pre, post) dense weights: lognormal E/I (sign by presyn) or dyadic
    synapse counts (geometric, mean 4) times 2**dy_exp."""
    mask = rng.random((n_pre, n_post)) < p
    exc = np.arange(n_pre) < int(round(exc_frac * n_pre))
    if dyadic:
        cnt = rng.geometric(0.25, size=(n_pre, n_post)).astype(np.float32)
        w = cnt * np.float32(2.0**dy_exp)
        w = np.where(exc[:, None], w, -w)
    else:
        w = rng.lognormal(-1.0, 1.0, size=(n_pre, n_post)).astype(np.float32) * np.float32(scale)
        w = np.where(exc[:, None], w, np.float32(inh_gain) * w)
    return (w * mask).astype(np.float32)


def canonical(conn):
    """Reference canonical COO (linear.py:278-292): the transposed matrix in
    sum_duplicates order.  Accepts a dense (pre, post) array or a scipy matrix."""
    import scipy.sparse as sp

    c = (sp.coo_array(conn) if isinstance(conn, np.ndarray) else conn.tocoo()).T
    c.sum_duplicates()
    return c.row.astype(np.int64), c.col.astype(np.int64), c.data.astype(np.float32)


def case_spmm(rng):
    import scipy.sparse as sp
    import torch
    from btorch.models.linear import SparseConn

    n_in, n_out, B = 300, 200, 5
    W = (rng.random((n_in, n_out)) < 0.1) * rng.standard_normal((n_in, n_out))
    W = W.astype(np.float32)
    m = SparseConn(sp.coo_array(W), enforce_dale=False, sparse_backend="native")
    x = (rng.random((B, n_in)) < 0.3) * rng.standard_normal((B, n_in))
    x = torch.tensor(x.astype(np.float32), requires_grad=True)
    out = m(x)
    g = torch.tensor(rng.standard_normal((B, n_out)).astype(np.float32))
    (out * g).sum().backward()
    return dict(
        post=m.indices[0].numpy(), src=m.indices[1].numpy(), w=m.magnitude.detach().numpy(),
        n_in=n_in, n_out=n_out, x=x.detach().numpy(), out=out.detach().numpy(), g=g.numpy(),
        grad_x=x.grad.numpy(), grad_w=m.magnitude.grad.numpy(),
    )


def _coef(tau, dt):
    """expm1(dt * lin) / lin with lin = -1.0 / tau, as the reference evaluates it."""
    import torch

    lin = -1.0 / torch.as_tensor(tau)
    return (torch.expm1(dt * lin) / lin).numpy().astype(np.float32)


def _run_rnn(neuron, synapse, inp, x, batch, names):
    """Run RecurrentNN; also returns the per-step outputs of the input module
    (recorded with a forward hook, i.e. exactly what the loop added to psc)."""
    import torch
    from btorch.models import environ
    from btorch.models.functional import init_net_state
    from btorch.models.rnn import RecurrentNN

    brain = RecurrentNN(neuron, synapse, neuron_inp_module=inp, update_state_names=names)
    init_net_state(brain, batch_size=batch, dtype=torch.float32)
    projected = []
    if inp is not None:
        inp.register_forward_hook(lambda m, a, out: projected.append(out.detach().clone()))
    with torch.no_grad(), environ.context(dt=1.0):
        z, states = brain(torch.tensor(x))
    proj = torch.stack(projected).numpy() if projected else None
    return brain, z.numpy(), {k: v.numpy() for k, v in states.items()}, proj


def case_lif(rng, *, n, p, batch, steps, dyadic, hard, tau_ref, c_in, in_gain, rate, scale=0.1):
    """LIF + ExponentialPSC(5) + SparseConn (+ DenseConn input if c_in)."""
    import scipy.sparse as sp
    import torch
    from btorch.models.linear import DenseConn, SparseConn
    from btorch.models.neurons import LIF
    from btorch.models.synapse import ExponentialPSC

    Wd = make_conn(rng, n, n, p, dyadic, scale=scale)
    conn = SparseConn(sp.coo_array(Wd), sparse_backend="native")
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=tau_ref, hard_reset=hard)
    syn = ExponentialPSC(n, tau_syn=5.0, linear=conn)
    if c_in:
        W_in = rng.normal(0.0, 0.05, size=(c_in, n)).astype(np.float32) * np.float32(in_gain)
        if dyadic:
            W_in = np.round(W_in * 64.0).astype(np.float32) / np.float32(64.0)
        inp = DenseConn(c_in, n, weight=torch.tensor(W_in))
        x = rng.poisson(rate, size=(steps, batch, c_in)).astype(np.float32)
    else:
        W_in = None
        inp = None
        x = (rng.poisson(rate, size=(steps, batch, n)) * in_gain).astype(np.float32)
        if dyadic:
            x = (np.round(x * 64.0) / 64.0).astype(np.float32)
    _, z, st, proj = _run_rnn(neuron, syn, inp, x, batch, ("neuron.v", "synapse.psc", "neuron.refractory"))
    post, src, w = canonical(Wd)
    out = dict(
        kind=0, n=n, batch=batch, hard=int(hard), use_ref=int(tau_ref is not None),
        tau_ref=np.float32(tau_ref or 0.0), tau=np.float32(20.0), vth=np.float32(1.0), vr=np.float32(0.0),
        cm=np.float32(1.0), psc_tau=np.float32(5.0), psc_coef=_coef(5.0, 1.0), dt=np.float32(1.0),
        post=post, src=src, w=w, n_bins=1, uniform_delay=0, x=x,
        z=np.packbits(z.astype(np.uint8), axis=-1, bitorder="little"), v=st["neuron.v"], psc=st["synapse.psc"],
    )
    if W_in is not None:
        out["W_in"] = W_in  # (c_in, n): DenseConn weight is W_in.T
        out["x_proj_ref"] = proj  # [steps, batch, n], the reference's own per-step projection
    return out


def case_alif(rng, *, n, p, batch, steps, dyadic):
    import scipy.sparse as sp
    from btorch.models.linear import SparseConn
    from btorch.models.neurons import ALIF
    from btorch.models.synapse import ExponentialPSC

    Wd = make_conn(rng, n, n, p, dyadic)
    conn = SparseConn(sp.coo_array(Wd), sparse_backend="native")
    neuron = ALIF(n, v_threshold=1.0, v_reset=0.0, c_m=1.0, g_leak=0.05, E_leak=0.0, E_k=-1.0,
                  tau_adapt=200.0, dg_k=0.07, tau_ref=2.0, hard_reset=True)
    syn = ExponentialPSC(n, tau_syn=5.0, linear=conn)
    x = (rng.poisson(0.08, size=(steps, batch, n)) * GAIN["alif"]).astype(np.float32)
    _, z, st, _ = _run_rnn(neuron, syn, None, x, batch, ("neuron.v", "synapse.psc", "neuron.g_k"))
    post, src, w = canonical(Wd)
    return dict(
        kind=1, n=n, batch=batch, hard=1, use_ref=1, tau_ref=np.float32(2.0), vth=np.float32(1.0),
        vr=np.float32(0.0), cm=np.float32(1.0), g_leak=np.float32(0.05), E_leak=np.float32(0.0),
        E_k=np.float32(-1.0), dg_k=np.float32(0.07), tau_adapt=np.float32(200.0), coef_gk=_coef(200.0, 1.0),
        psc_tau=np.float32(5.0), psc_coef=_coef(5.0, 1.0), dt=np.float32(1.0),
        post=post, src=src, w=w, n_bins=1, uniform_delay=0, x=x,
        z=np.packbits(z.astype(np.uint8), axis=-1, bitorder="little"), v=st["neuron.v"],
        psc=st["synapse.psc"], g_k=st["neuron.g_k"],
    )


def case_delayed(rng, *, n, p, batch, steps, D):
    """LIF + DelayedPSC(ExponentialPSC, max_delay_steps=D), dyadic weights."""
    import scipy.sparse as sp
    from btorch.models.linear import SparseConn
    from btorch.models.neurons import LIF
    from btorch.models.synapse import DelayedPSC, ExponentialPSC

    Wd = make_conn(rng, n, n, p, True)
    conn = SparseConn(sp.coo_array(Wd), sparse_backend="native")
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True)
    syn = DelayedPSC(ExponentialPSC(n, tau_syn=5.0, linear=conn), max_delay_steps=D, use_circular_buffer=True)
    x = (np.round(rng.poisson(0.1, size=(steps, batch, n)) * GAIN["delay"] * 64) / 64).astype(np.float32)
    _, z, st, _ = _run_rnn(neuron, syn, None, x, batch, ("neuron.v", "synapse.psc_module.psc"))
    post, src, w = canonical(Wd)
    return dict(
        kind=0, n=n, batch=batch, hard=1, use_ref=1, tau_ref=np.float32(2.0), tau=np.float32(20.0),
        vth=np.float32(1.0), vr=np.float32(0.0), cm=np.float32(1.0), psc_tau=np.float32(5.0),
        psc_coef=_coef(5.0, 1.0), dt=np.float32(1.0), post=post, src=src, w=w, n_bins=1, uniform_delay=D,
        x=x, z=np.packbits(z.astype(np.uint8), axis=-1, bitorder="little"), v=st["neuron.v"],
        psc=st["synapse.psc_module.psc"],
    )


def case_hetero(rng, *, n, p, batch, steps, D):
    """LIF + HeterSynapsePSC(n_receptor=1, ExponentialPSC, max_delay_steps=D) on
    a delay-expanded matrix from expand_conn_for_delays (per-synapse delays)."""
    import pandas as pd
    import scipy.sparse as sp
    from btorch.connectome.connection import expand_conn_for_delays
    from btorch.models.linear import SparseConn
    from btorch.models.neurons import LIF
    from btorch.models.synapse import ExponentialPSC, HeterSynapsePSC

    Wd = make_conn(rng, n, n, p, True)
    base = sp.coo_array(Wd)
    delays = rng.integers(1, D + 1, size=base.nnz)  # 1..D steps
    conn_d = expand_conn_for_delays(base, delays - 1, n_delay_bins=D)
    conn = SparseConn(conn_d, sparse_backend="native")
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True)
    rti = pd.DataFrame({"receptor_type": ["syn"], "receptor_index": [0]})
    syn = HeterSynapsePSC(n, n_receptor=1, receptor_type_index=rti, linear=conn, base_psc=ExponentialPSC,
                          max_delay_steps=D, use_circular_buffer=True, tau_syn=5.0)
    x = (np.round(rng.poisson(0.1, size=(steps, batch, n)) * GAIN["delay"] * 64) / 64).astype(np.float32)
    _, z, st, _ = _run_rnn(neuron, syn, None, x, batch, ("neuron.v", "synapse.psc"))
    post, src, w = canonical(conn_d)
    return dict(
        kind=0, n=n, batch=batch, hard=1, use_ref=1, tau_ref=np.float32(2.0), tau=np.float32(20.0),
        vth=np.float32(1.0), vr=np.float32(0.0), cm=np.float32(1.0), psc_tau=np.float32(5.0),
        psc_coef=_coef(5.0, 1.0), dt=np.float32(1.0), post=post, src=src, w=w, n_bins=D, uniform_delay=0,
        x=x, z=np.packbits(z.astype(np.uint8), axis=-1, bitorder="little"), v=st["neuron.v"], psc=st["synapse.psc"],
    )


TRACE_STEPS = 40
GAIN = {"c1": 1.0, "soft": 0.6, "inp": 4.0, "alif": 0.6, "delay": 0.5}


def case_train(rng, *, n, p, batch, steps, windows, c_in, n_out, spiking, chunk, unroll):
    """Truncated-BPTT training windows: LIF (sigmoid surrogate, alpha 5) +
    ExponentialPSC + SparseConn, DenseConn input, linear readout of the spikes
    to sinusoid targets, MSE; RecurrentNN with grad_checkpoint over chunks.
    Per window: forward, backward, gradients recorded, detach_net (no
    optimizer step, so every window uses the same weights).

    The backward recomputes the checkpointed chunks through RecurrentNN's
    _pure (rnn.py:187-195), which rebinds the module state to each chunk's
    recomputation, and torch's non-reentrant checkpoint may stop a
    recomputation early -- so after backward the reference's modules hold a
    state that depends on autograd internals.  The forward's final state is
    therefore saved before backward and restored after it, which is the
    state truncated BPTT continues from."""
    import scipy.sparse as sp
    import torch
    from btorch.models import environ
    from btorch.models.functional import detach_net, init_net_state, named_hidden_states, set_hidden_states
    from btorch.models.linear import DenseConn, SparseConn
    from btorch.models.neurons import LIF
    from btorch.models.rnn import RecurrentNN
    from btorch.models.surrogate import Sigmoid
    from btorch.models.synapse import ExponentialPSC

    Wd = make_conn(rng, n, n, p, dyadic=True, dy_exp=-6)
    conn = SparseConn(sp.coo_array(Wd), sparse_backend="native")
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True,
                 surrogate_function=Sigmoid(alpha=5.0, spiking=spiking))
    syn = ExponentialPSC(n, tau_syn=5.0, linear=conn)
    W_in = (np.round(rng.normal(0.0, 0.3, size=(c_in, n)) * 64.0) / 64.0).astype(np.float32)
    inp = DenseConn(c_in, n, weight=torch.tensor(W_in))
    W_out = (np.round(rng.normal(0.0, 0.5, size=(n_out, n)) * 64.0) / 64.0).astype(np.float32)
    b_out = (np.round(rng.normal(0.0, 0.5, size=n_out) * 64.0) / 64.0).astype(np.float32)
    readout = torch.nn.Linear(n, n_out)
    with torch.no_grad():
        readout.weight.copy_(torch.tensor(W_out))
        readout.bias.copy_(torch.tensor(b_out))
    brain = RecurrentNN(neuron, syn, neuron_inp_module=inp, update_state_names=("neuron.v",),
                        grad_checkpoint=True, chunk_size=chunk, unroll=unroll)
    init_net_state(brain, batch_size=batch, dtype=torch.float32)
    T = steps * windows
    x = rng.poisson(0.3, size=(T, batch, c_in)).astype(np.float32)
    freq = rng.uniform(1.0, 20.0, size=(1, batch, n_out))
    phase = rng.uniform(0.0, 2 * np.pi, size=(1, batch, n_out))
    t = np.arange(T, dtype=np.float64)[:, None, None]
    target = np.sin(2 * np.pi * freq * t * 1e-3 + phase).astype(np.float32)
    out = dict(n=n, batch=batch, steps=steps, windows=windows, c_in=c_in, n_out=n_out, spiking=int(spiking),
               chunk=chunk, unroll=unroll, tau=np.float32(20.0), tau_ref=np.float32(2.0), alpha=np.float32(5.0),
               psc_tau=np.float32(5.0), W_in=W_in, W_out=W_out, b_out=b_out, x=x, target=target)
    post, src, w = canonical(Wd)
    out.update(post=post, src=src, w=w)
    assert np.array_equal(conn.indices[0].numpy(), post) and np.array_equal(conn.indices[1].numpy(), src)
    zs, losses = [], []
    with environ.context(dt=1.0):
        for k in range(windows):
            sl = slice(k * steps, (k + 1) * steps)
            z, _ = brain(torch.tensor(x[sl]))
            y = readout(z)
            loss = ((y - torch.tensor(target[sl])) ** 2).mean()
            final = dict(named_hidden_states(brain))
            for m in (brain, readout):
                m.zero_grad(set_to_none=True)
            loss.backward()
            set_hidden_states(brain, final)
            out[f"grad_w_{k}"] = conn.magnitude.grad.numpy().copy()
            out[f"grad_win_{k}"] = inp.weight.grad.numpy().copy()  # (n, c_in) like DenseConn.weight
            out[f"grad_wout_{k}"] = readout.weight.grad.numpy().copy()
            out[f"grad_bout_{k}"] = readout.bias.grad.numpy().copy()
            losses.append(float(loss.detach()))
            zs.append(z.detach().numpy())
            detach_net(brain)
    out["loss"] = np.array(losses, np.float32)
    out["z"] = np.packbits(np.concatenate(zs).astype(np.uint8) if spiking else (np.concatenate(zs) > 0.5),
                           axis=-1, bitorder="little")
    return out


def case_fp64(rng, *, n, p, steps, c_in, rate, scale, in_gain):
    """The C1 configuration's model (LIF tau 20, refractory 2, hard reset,
    ExponentialPSC 5, lognormal E/I SparseConn, DenseConn input from Poisson
    channels, batch 1) at a reduced size with C1's in-degree (82) and active
    input channels per step (10), run by the reference twice on the same
    inputs: in fp32 and in fp64 (dtype=torch.float64 on every module and the
    state).  The fp64 membrane trace is the yardstick for the fp32 error of
    the first `steps` steps: per-step max |v32 - v64| over all neurons and the
    first raster divergence are stored, with the traces of 64 neurons."""
    import scipy.sparse as sp
    import torch
    from btorch.models import environ
    from btorch.models.functional import init_net_state
    from btorch.models.linear import DenseConn, SparseConn
    from btorch.models.neurons import LIF
    from btorch.models.rnn import RecurrentNN
    from btorch.models.synapse import ExponentialPSC

    Wd = make_conn(rng, n, n, p, dyadic=False, scale=scale)
    W_in = (rng.normal(0.0, 0.05, size=(c_in, n)) * in_gain).astype(np.float32)
    x = rng.poisson(rate, size=(steps, 1, c_in)).astype(np.float32)
    out = {}
    for dt_name, dtype in (("32", torch.float32), ("64", torch.float64)):
        conn = SparseConn(sp.coo_array(Wd.astype(np.float64) if dtype == torch.float64 else Wd),
                          sparse_backend="native", dtype=dtype)
        neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True, dtype=dtype)
        syn = ExponentialPSC(n, tau_syn=5.0, linear=conn)
        inp = DenseConn(c_in, n, weight=torch.tensor(W_in, dtype=dtype), dtype=dtype)
        brain = RecurrentNN(neuron, syn, neuron_inp_module=inp, update_state_names=("neuron.v",))
        init_net_state(brain, batch_size=1, dtype=dtype)
        with torch.no_grad(), environ.context(dt=1.0):
            z, st = brain(torch.tensor(x, dtype=dtype))
        out["v" + dt_name] = st["neuron.v"].numpy()
        out["z" + dt_name] = np.packbits(z.numpy().astype(np.uint8), axis=-1, bitorder="little")
    post, src, w = canonical(Wd)
    z32 = np.unpackbits(out["z32"], axis=-1, bitorder="little")[..., :n]
    z64 = np.unpackbits(out["z64"], axis=-1, bitorder="little")[..., :n]
    bad = np.nonzero((z32 != z64).reshape(steps, -1).any(1))[0]
    k = int(bad[0]) if bad.size else steps
    err = np.abs(out["v32"].astype(np.float64) - out["v64"]).reshape(steps, -1)
    keep = slice(0, 64)  # traces of the first 64 neurons; error statistics over all
    out.update(n=n, batch=1, x=x, W_in=W_in, post=post.astype(np.int32), src=src.astype(np.int32), w=w,
               steps=steps, first_divergence=k, err_max=err.max(axis=1),
               v32=out["v32"][:, :, keep], v64=out["v64"][:, :, keep])
    return out


def case_constrained(rng):
    """SparseConstrainedConn (3 groups) forward and backward on graded inputs,
    with non-unit group magnitudes."""
    import scipy.sparse as sp
    import torch
    from btorch.models.linear import SparseConstrainedConn

    n_in, n_out, B, G = 120, 90, 4, 3
    W = ((rng.random((n_in, n_out)) < 0.15) * rng.standard_normal((n_in, n_out))).astype(np.float32)
    Wc = sp.coo_array(W)
    C = sp.coo_array((rng.integers(1, G + 1, size=Wc.nnz).astype(np.float32), (Wc.row, Wc.col)), shape=W.shape)
    m = SparseConstrainedConn(Wc, C, sparse_backend="native")
    mag = np.array([0.5, 1.25, 2.0], np.float32)
    with torch.no_grad():
        m.magnitude.copy_(torch.tensor(mag))
    x = torch.tensor(((rng.random((B, n_in)) < 0.3) * rng.standard_normal((B, n_in))).astype(np.float32),
                     requires_grad=True)
    out = m(x)
    g = torch.tensor(rng.standard_normal((B, n_out)).astype(np.float32))
    (out * g).sum().backward()
    return dict(n_in=n_in, n_out=n_out, W=W, C_row=C.row.astype(np.int64), C_col=C.col.astype(np.int64),
                C_data=C.data, magnitude=mag, x=x.detach().numpy(), out=out.detach().numpy(), g=g.numpy(),
                grad_x=x.grad.numpy(), grad_mag=m.magnitude.grad.numpy(),
                group=m._constraint_scatter_indices.numpy())


def case_receptors(rng, *, n, p, batch, steps, n_rec):
    """LIF + HeterSynapsePSC with n_rec receptors (ExponentialPSC base, a time
    constant per receptor), no delays: the connection maps presynaptic
    neurons to (post, receptor) pairs, flat index post * n_rec + receptor."""
    import pandas as pd
    import scipy.sparse as sp
    import torch
    from btorch.models.linear import SparseConn
    from btorch.models.neurons import LIF
    from btorch.models.synapse import ExponentialPSC, HeterSynapsePSC

    Wd = make_conn(rng, n, n * n_rec, p, dyadic=True, dy_exp=-6)
    conn = SparseConn(sp.coo_array(Wd), sparse_backend="native")
    taus = np.array([5.0, 20.0, 2.0, 10.0][:n_rec], np.float32)
    rti = pd.DataFrame({"receptor_type": [f"r{r}" for r in range(n_rec)], "receptor_index": list(range(n_rec))})
    syn = HeterSynapsePSC(n, n_rec, rti, conn, base_psc=ExponentialPSC,
                          tau_syn=torch.tensor(np.tile(taus, n)))
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True)
    x = (np.round(rng.poisson(0.06, size=(steps, batch, n)) * 0.75 * 64) / 64).astype(np.float32)
    _, z, st, _ = _run_rnn(neuron, syn, None, x, batch, ("neuron.v", "synapse.psc", "synapse.base_psc.psc"))
    post, src, w = canonical(Wd)
    return dict(n=n, batch=batch, n_rec=n_rec, taus=taus, post=post, src=src, w=w, x=x,
                z=np.packbits(z.astype(np.uint8), axis=-1, bitorder="little"), v=st["neuron.v"],
                psc=st["synapse.psc"], psc_rec=st["synapse.base_psc.psc"])



def connectome_tables(rng, n, n_conn, nan_ids=(), dup=True):
    """Seeded neuron and connection tables in the reference's column layout
    (simple_id, EI; pre/post_simple_id, syn_count, delay_steps, nt)."""
    import pandas as pd

    ei = rng.choice(np.array(["E", "I"], dtype=object), size=n, p=[0.7, 0.3])
    ei[list(nan_ids)] = np.nan
    neurons = pd.DataFrame({"simple_id": np.arange(n), "root_id": 1000 + np.arange(n), "EI": ei})
    pre = rng.integers(0, n, n_conn)
    post = rng.integers(0, n, n_conn)
    if not dup:
        key = np.unique(pre * n + post)
        key = rng.permutation(key)
        pre, post = key // n, key % n
    conns = pd.DataFrame({"pre_simple_id": pre, "post_simple_id": post,
                          "syn_count": rng.integers(1, 10, len(pre)),
                          "delay_steps": rng.integers(0, 8, len(pre)),
                          "nt": rng.choice(np.array(["ach", "gaba", "glut"], dtype=object), size=len(pre))})
    return neurons, conns


def _save_coo(out, name, m):
    m = m.tocoo()
    out[f"{name}.row"] = np.asarray(m.row, np.int64)
    out[f"{name}.col"] = np.asarray(m.col, np.int64)
    out[f"{name}.data"] = np.asarray(m.data)
    out[f"{name}.shape"] = np.asarray(m.shape, np.int64)


def case_connectome_format(rng):
    """make_hetersynapse_conn / stack_hetersynapse outputs (entries in the
    reference's own order) on seeded tables, every mode the reference has."""
    import json
    import warnings

    from btorch.connectome.connection import make_hetersynapse_conn, stack_hetersynapse

    out = {}
    tables = {"dup": connectome_tables(rng, 60, 500, nan_ids=(3, 17, 41)),
              "uniq": connectome_tables(rng, 50, 400, dup=False)}
    for t, (neu, con) in tables.items():
        for c in neu.columns:
            out[f"in.{t}.neurons.{c}"] = neu[c].to_numpy().astype(str if c == "EI" else np.int64)
        for c in con.columns:
            out[f"in.{t}.conns.{c}"] = con[c].to_numpy().astype(str if c == "nt" else np.int64)
    neu_nan, con_dup = tables["dup"]
    neu_ok = neu_nan.copy()
    neu_ok.loc[neu_ok.EI.isna(), "EI"] = "E"
    neu_u, con_u = tables["uniq"]
    runs = {
        "neuron": (neu_ok, con_dup, dict()),
        "neuron_ignore_post": (neu_ok, con_dup, dict(ignore_post_type=True)),
        "neuron_delay": (neu_ok, con_dup, dict(delay_col="delay_steps", n_delay_bins=5)),
        "neuron_filter": (neu_nan, con_dup, dict(dropna="filter")),
        "neuron_unknown": (neu_nan, con_dup, dict(dropna="unknown")),
        "neuron_filter_ignore_post": (neu_nan, con_dup, dict(dropna="filter", ignore_post_type=True)),
        "connection": (neu_ok, con_dup, dict(receptor_type_col="nt", receptor_type_mode="connection")),
        "connection_delay": (neu_u, con_u, dict(receptor_type_col="nt", receptor_type_mode="connection",
                                                delay_col="delay_steps", n_delay_bins=6)),
        "delay_only": (neu_ok, con_dup, dict(receptor_type_col=None, delay_col="delay_steps", n_delay_bins=4)),
    }
    for name, (neu, con, kw) in runs.items():
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            m, idx = make_hetersynapse_conn(neu, con, **kw)
        _save_coo(out, name, m)
        out[f"{name}.index"] = np.array(idx.to_json(orient="split"))
        out[f"{name}.kwargs"] = np.array(json.dumps(kw))
    for mode, kw in (("dict_neuron", dict()), ("dict_connection", dict(receptor_type_col="nt",
                                                                      receptor_type_mode="connection"))):
        d, idx = make_hetersynapse_conn(neu_ok, con_dup, return_dict=True, **kw)
        out[f"{mode}.keys"] = np.array(json.dumps([list(k) if isinstance(k, tuple) else k for k in d]))
        for i, m in enumerate(d.values()):
            _save_coo(out, f"{mode}.{i}", m)
        out[f"{mode}.index"] = np.array(idx.to_json(orient="split"))
        for how in ("pre", "post", "all"):
            m2, idx2 = stack_hetersynapse(d, idx, ignore_receptor_type=how)
            _save_coo(out, f"{mode}.collapse_{how}", m2)
            out[f"{mode}.collapse_{how}.index"] = np.array(idx2.to_json(orient="split"))
        _save_coo(out, f"{mode}.stacked", stack_hetersynapse(d, idx))
    return out


def case_receptors_delay(rng, *, n, n_conn, batch, steps, D):
    """LIF + HeterSynapsePSC(n_receptor=4 E/I pairs, ExponentialPSC with a time
    constant per receptor, max_delay_steps=D) on the matrix
    make_hetersynapse_conn(..., delay_col, n_delay_bins=D) builds from seeded
    tables; weights syn_count * 2**-5, negative from inhibitory neurons."""
    import scipy.sparse as sp
    import torch
    from btorch.connectome.connection import make_hetersynapse_conn
    from btorch.models.linear import SparseConn
    from btorch.models.neurons import LIF
    from btorch.models.synapse import ExponentialPSC, HeterSynapsePSC

    neu, con = connectome_tables(rng, n, n_conn)
    m, idx = make_hetersynapse_conn(neu, con, delay_col="delay_steps", n_delay_bins=D)
    m = m.tocoo()
    inh = (neu.EI.to_numpy() == "I")[m.row // D]
    w = (m.data * 2.0**-5 * np.where(inh, -1.0, 1.0)).astype(np.float32)
    W = sp.coo_array((w, (m.row, m.col)), shape=m.shape)
    conn = SparseConn(W, sparse_backend="native")
    n_rec = len(idx)
    taus = np.array([5.0, 3.0, 10.0, 2.5][:n_rec], np.float32)
    syn = HeterSynapsePSC(n, n_rec, idx, conn, base_psc=ExponentialPSC, max_delay_steps=D,
                          use_circular_buffer=True, tau_syn=torch.tensor(np.tile(taus, n)))
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True)
    x = (np.round(rng.poisson(0.08, size=(steps, batch, n)) * 0.75 * 64) / 64).astype(np.float32)
    _, z, st, _ = _run_rnn(neuron, syn, None, x, batch, ("neuron.v", "synapse.psc", "synapse.base_psc.psc"))
    post, src, wc = canonical(W)
    out = dict(n=n, batch=batch, n_rec=n_rec, n_bins=D, taus=taus, post=post, src=src, w=wc, x=x,
               z=np.packbits(z.astype(np.uint8), axis=-1, bitorder="little"), v=st["neuron.v"],
               psc=st["synapse.psc"], psc_rec=st["synapse.base_psc.psc"])
    for c in neu.columns:
        out[f"neurons.{c}"] = neu[c].to_numpy().astype(str if c == "EI" else np.int64)
    for c in con.columns:
        out[f"conns.{c}"] = con[c].to_numpy().astype(str if c == "nt" else np.int64)
    return out


def constraint_tables(rng, n, n_conn):
    """Seeded tables with cell types (three missing), two cell-type columns,
    root ids (every 7th connection names a root id absent from the neuron
    table) and duplicate (pre, post) rows."""
    import pandas as pd

    ct = rng.choice(np.array(["a", "b", "c", "d"], dtype=object), size=n)
    ct[[2, 9, 30]] = np.nan
    neurons = pd.DataFrame({"root_id": 1000 + np.arange(n), "simple_id": np.arange(n), "cell_type": ct,
                            "EI": rng.choice(np.array(["E", "I"], dtype=object), size=n, p=[0.7, 0.3]),
                            "ct2": rng.choice(np.array(["x", "y"], dtype=object), size=n)})
    pre = rng.integers(0, n, n_conn)
    post = rng.integers(0, n, n_conn)
    conns = pd.DataFrame({"pre_simple_id": pre, "post_simple_id": post, "pre_root_id": 1000 + pre,
                          "post_root_id": 1000 + post, "syn_count": rng.integers(1, 9, n_conn),
                          "nt": rng.choice(np.array(["ach", "gaba", "glut"], dtype=object), size=n_conn)})
    conns.loc[::7, "pre_root_id"] = 99999
    return neurons, conns


CONSTRAINT_RUNS = [
    dict(constraint_mode=m, receptor_type_mode=r, ignore_post_type=i, nan_in_same_group=g, cell_type_col=c)
    for m in ("full", "cell_only", "cell_and_receptor") for r in ("neuron", "connection")
    for i in (False, True) for g in (True, False) for c in ("cell_type", "ct2")]


def case_connectome_constraint(rng):
    """make_constraint_by_neuron_type / make_hetersynapse_constraint /
    make_hetersynapse_constrained_conn outputs on seeded tables, every mode."""
    import json

    from btorch.connectome.connection import (make_constraint_by_neuron_type,
                                              make_hetersynapse_constrained_conn,
                                              make_hetersynapse_constraint)

    neu, con = constraint_tables(rng, 60, 500)
    out = {}
    for c in neu.columns:
        out[f"in.neurons.{c}"] = neu[c].to_numpy().astype(np.int64 if neu[c].dtype.kind == "i" else str)
    for c in con.columns:
        out[f"in.conns.{c}"] = con[c].to_numpy().astype(np.int64 if con[c].dtype.kind == "i" else str)
    for g in (True, False):
        _save_coo(out, f"by_type.{int(g)}", make_constraint_by_neuron_type(neu, con, nan_in_same_group=g))
    for i, kw in enumerate(CONSTRAINT_RUNS):
        kw = dict(kw, receptor_type_col="EI" if kw["receptor_type_mode"] == "neuron" else "nt")
        _save_coo(out, f"hetero.{i}", make_hetersynapse_constraint(neu, con, **kw))
        out[f"hetero.{i}.kwargs"] = np.array(json.dumps(kw))
    import torch
    from btorch.models.linear import SparseConstrainedConn

    for mode in ("cell_only", "cell_and_receptor"):
        m, c, idx = make_hetersynapse_constrained_conn(neu, con, constraint_mode=mode)
        _save_coo(out, f"combined.{mode}.conn", m)
        _save_coo(out, f"combined.{mode}.constraint", c)
        out[f"combined.{mode}.index"] = np.array(idx.to_json(orient="split"))
        lin = SparseConstrainedConn.from_hetersynapse(m.astype(np.float32), c, idx, enforce_dale=True)
        out[f"combined.{mode}.group"] = lin._constraint_scatter_indices.numpy().astype(np.int64)
        out[f"combined.{mode}.n_groups"] = np.int64(lin.magnitude.numel())
        # the inspection helpers after two magnitude edits
        with torch.no_grad():
            lin.magnitude.copy_(torch.linspace(0.5, 1.5, lin.magnitude.numel()))
        lin.set_group_magnitude(group_id=1, value=2.5)
        lin.set_group_magnitude(receptor_pair=("E", "I"), value=0.25)
        out[f"combined.{mode}.group_info"] = np.array(lin.get_group_info(include_weights=True).to_json(
            orient="split", double_precision=15))
        wbg = lin.get_weights_by_group()
        out[f"combined.{mode}.by_group_len"] = np.array([len(wbg[g]) for g in sorted(wbg)], np.int64)
        out[f"combined.{mode}.by_group"] = np.concatenate([wbg[g].detach().numpy() for g in sorted(wbg)])
    return out


STATE_DICT_MODULES = [
    ("LIF", dict(n_neuron=8)),
    ("LIF", dict(n_neuron=8, tau=[10.0 + 2.5 * i for i in range(8)], v_threshold=[1.5] * 8, tau_ref=2.0,
                 trainable_param=["tau"])),
    ("ALIF", dict(n_neuron=8, tau_adapt=[50.0 + 5 * i for i in range(8)], dg_k=0.3)),
    ("ExponentialPSC", dict(n_neuron=8, tau_syn=[5.0 + i for i in range(8)])),
]


def _module_kwargs(kw):
    """JSON-able constructor arguments -> the module's (lists of per-neuron
    values become tensors, trainable_param a set)."""
    import torch

    out = {}
    for k, v in kw.items():
        if k == "trainable_param":
            out[k] = set(v)
        elif isinstance(v, list):
            out[k] = torch.tensor(v, dtype=torch.float32)
        else:
            out[k] = v
    return out


def case_state_dict(rng):
    """state_dicts of the reference's LIF / ALIF / ExponentialPSC for scalar,
    uniform and per-neuron parameters, and the parameter shapes after loading
    a checkpoint into a module built with other values."""
    import json

    import torch
    from btorch.models.neurons import ALIF, LIF
    from btorch.models.synapse import ExponentialPSC

    classes = {"LIF": LIF, "ALIF": ALIF,
               "ExponentialPSC": lambda **kw: ExponentialPSC(linear=torch.nn.Identity(), **kw)}
    out = {"modules": np.array(json.dumps(STATE_DICT_MODULES))}
    for i, (cls, kw) in enumerate(STATE_DICT_MODULES):
        m = classes[cls](**_module_kwargs(kw))
        sd = m.state_dict()
        out[f"m{i}.keys"] = np.array(json.dumps(list(sd)))
        for k, v in sd.items():
            out[f"m{i}.{k}"] = v.detach().numpy()
        # into a module built with the defaults: which shapes the checkpoint gives
        fresh = classes[cls](n_neuron=8, **({"tau_syn": 5.0} if cls == "ExponentialPSC" else {}))
        fresh.load_state_dict(sd, strict=False)
        out[f"m{i}.reloaded"] = np.array(json.dumps({k: list(v.shape) for k, v in fresh.state_dict(keep_vars=True).items()}))
    # a full uniform value collapses to a scalar, a non-uniform one expands
    lif = LIF(n_neuron=8)
    lif.load_state_dict({"tau": torch.full((8,), 25.0)}, strict=False)
    out["uniform_tau_shape"] = np.array(list(lif.tau.shape), np.int64)
    lif.load_state_dict({"tau": torch.arange(8.0) + 1}, strict=False)
    out["nonuniform_tau_shape"] = np.array(list(lif.tau.shape), np.int64)
    return out


SURROGATE_RUNS = [dict(alpha=a, damping_factor=d, spiking=sp)
                  for a in (2.0, 5.0, 0.7) for d in (1.0, 0.3) for sp in (True, False)]


def case_surrogate(rng):
    """The reference's Sigmoid surrogate called directly: forward and the
    gradient of sum(forward * r) on a seeded grid around the threshold."""
    import json

    import torch
    from btorch.models.surrogate import Sigmoid

    x = np.concatenate([np.linspace(-3, 3, 601), rng.standard_normal(400) * 2, [0.0, -0.0]]).astype(np.float32)
    r = rng.standard_normal(x.size).astype(np.float32)
    out = {"x": x, "r": r, "runs": np.array(json.dumps(SURROGATE_RUNS))}
    for i, kw in enumerate(SURROGATE_RUNS):
        xt = torch.tensor(x, requires_grad=True)
        y = Sigmoid(**kw)(xt)
        (y * torch.tensor(r)).sum().backward()
        out[f"y{i}"] = y.detach().numpy()
        out[f"g{i}"] = xt.grad.numpy()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("BTORCH_REFERENCE"),
                    help="reference checkout (default: $BTORCH_REFERENCE)")
    ap.add_argument("--only", default="", help="comma-separated case names (default: all)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or BTORCH_REFERENCE")
    _import_reference(args.ref)
    import torch

    torch.set_num_threads(4)
    cases = {
        "spmm_graded": lambda r: case_spmm(r),
        "lif_c1_small": lambda r: case_lif(r, n=512, p=0.02 * 8, batch=1, steps=150, dyadic=False, hard=True,
                                           tau_ref=2.0, c_in=128, in_gain=GAIN["c1"], rate=0.05,
                                           scale=0.01),
        "lif_dyadic_soft": lambda r: case_lif(r, n=256, p=0.05, batch=4, steps=120, dyadic=True, hard=False,
                                              tau_ref=None, c_in=0, in_gain=GAIN["soft"], rate=0.05),
        "lif_dyadic_input": lambda r: case_lif(r, n=256, p=0.05, batch=3, steps=120, dyadic=True, hard=True,
                                               tau_ref=2.0, c_in=64, in_gain=GAIN["inp"], rate=0.05),
        "alif_exppsc": lambda r: case_alif(r, n=320, p=0.05, batch=3, steps=150, dyadic=False),
        "delayed_psc": lambda r: case_delayed(r, n=256, p=0.05, batch=2, steps=120, D=3),
        "hetero_delay": lambda r: case_hetero(r, n=256, p=0.05, batch=2, steps=120, D=6),
        "train_spiking": lambda r: case_train(r, n=96, p=0.1, batch=3, steps=30, windows=2, c_in=16, n_out=4,
                                              spiking=True, chunk=10, unroll=5),
        "train_smooth": lambda r: case_train(r, n=96, p=0.1, batch=3, steps=30, windows=2, c_in=16, n_out=4,
                                             spiking=False, chunk=10, unroll=5),
        "fp64_c1": lambda r: case_fp64(r, n=1024, p=0.08, steps=200, c_in=250, rate=0.04, scale=0.01,
                                       in_gain=GAIN["c1"]),
        "constrained_spmm": lambda r: case_constrained(r),
        "receptors2": lambda r: case_receptors(r, n=200, p=0.03, batch=3, steps=100, n_rec=2),
        "connectome_format": lambda r: case_connectome_format(r),
        "receptors_delay": lambda r: case_receptors_delay(r, n=300, n_conn=9000, batch=3, steps=120, D=5),
        "connectome_constraint": lambda r: case_connectome_constraint(r),
        "state_dict": lambda r: case_state_dict(r),
        "surrogate": lambda r: case_surrogate(r),
    }
    only = set(args.only.split(",")) if args.only else None
    for i, (name, fn) in enumerate(cases.items()):
        if only is not None and name not in only:
            continue
        rng = np.random.default_rng(1000 + i)
        d = fn(rng)
        # Full spike rasters (bit-packed) are kept; float traces only for the
        # first TRACE_STEPS steps, plus the state after the last step.
        for key in ("v", "psc", "g_k", "psc_rec"):
            if key in d and "z" in d and d[key].ndim == 3:
                d[key + "_final"] = d[key][-1]
                d[key] = d[key][:TRACE_STEPS]
        np.savez_compressed(OUT / f"{name}.npz", **d)
        extra = ""
        if "z" in d:
            z = np.unpackbits(d["z"], axis=-1, bitorder="little")[..., : d["n"]]
            extra = f" rate/step={z.mean():.4f}"
        print(f"{name}: saved{extra}")


if __name__ == "__main__":
    main()
