"""Surrogate-gradient BPTT through the hand-written backward kernels.

* Against the reference's own autograd (tests/golden/train_*.npz, made by
  make_golden.py from the reference on the CPU): truncated-BPTT windows with
  checkpointed chunks, LIF + ExponentialPSC + SparseConn + DenseConn input,
  linear readout, MSE -- loss and every parameter gradient within 1e-4
  relative (norm-wise), spike rasters identical.
* Against finite differences of the smooth-surrogate forward (sigmoid spikes).

Both training paths are checked: the per-module one (an autograd node per
module per step) and the fused BPTT (one autograd Function per call,
btorch_b200/models/bptt.py).
"""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from btorch_b200.models import LIF, DenseConn, ExponentialPSC, RecurrentNN, Sigmoid, SparseConn, environ
from btorch_b200.models.functional import detach_net, init_net_state
from tests import cases

pytestmark = pytest.mark.gpu
DEV = "cuda"


def build(d, direction="gather", refractory=True, alpha=None, fused=True):
    n = int(d["n"])
    W = sp.coo_array((d["w"], (d["src"], d["post"])), shape=(n, n))
    conn = SparseConn(W, sparse_config={"direction": direction})
    tau_ref = float(d["tau_ref"]) if refractory else None
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=float(d["tau"]), tau_ref=tau_ref, hard_reset=True,
                 surrogate_function=Sigmoid(alpha=float(d["alpha"]) if alpha is None else alpha,
                                            spiking=bool(d["spiking"])))
    syn = ExponentialPSC(n, tau_syn=float(d["psc_tau"]), linear=conn)
    inp = DenseConn(int(d["c_in"]), n, weight=torch.tensor(d["W_in"]))
    brain = RecurrentNN(neuron, syn, neuron_inp_module=inp, update_state_names=("neuron.v",), grad_checkpoint=True,
                        chunk_size=int(d["chunk"]), unroll=int(d["unroll"]), fused=fused).to(DEV)
    readout = torch.nn.Linear(n, int(d["n_out"])).to(DEV)
    with torch.no_grad():
        readout.weight.copy_(torch.tensor(d["W_out"]))
        readout.bias.copy_(torch.tensor(d["b_out"]))
    init_net_state(brain, batch_size=int(d["batch"]), dtype=torch.float32, device=DEV)
    return brain, readout, conn, inp


def train_windows(d, direction="gather", fused=True):
    brain, readout, conn, inp = build(d, direction, fused=fused)
    steps, windows = int(d["steps"]), int(d["windows"])
    x = torch.tensor(d["x"], device=DEV)
    target = torch.tensor(d["target"], device=DEV)
    out = {"loss": [], "z": []}
    with environ.context(dt=1.0):
        for k in range(windows):
            sl = slice(k * steps, (k + 1) * steps)
            z, st = brain(x[sl])
            assert brain.last_path == ("fused-bptt" if fused else "modular"), brain.last_path
            assert st["neuron.v"].shape == (steps, int(d["batch"]), int(d["n"]))
            loss = ((readout(z) - target[sl]) ** 2).mean()
            for m in (brain, readout):
                m.zero_grad(set_to_none=True)
            loss.backward()
            out[f"grad_w_{k}"] = conn.magnitude.grad.cpu().numpy()
            out[f"grad_win_{k}"] = inp.weight.grad.cpu().numpy()
            out[f"grad_wout_{k}"] = readout.weight.grad.cpu().numpy()
            out[f"grad_bout_{k}"] = readout.bias.grad.cpu().numpy()
            out["loss"].append(float(loss.detach()))
            out["z"].append(z.detach().cpu().numpy())
            detach_net(brain)
    return out


def rel_err(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / max(np.linalg.norm(b.astype(np.float64)), 1e-30))


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("direction", ["gather", "scatter"])
@pytest.mark.parametrize("name", ["train_spiking", "train_smooth"])
def test_bptt_gradients_match_reference_autograd(name, direction, fused):
    d = cases.load(name)
    out = train_windows(d, direction, fused)
    n = int(d["n"])
    z = np.concatenate(out["z"])
    if int(d["spiking"]):
        ref_z = np.unpackbits(d["z"], axis=-1, bitorder="little")[..., :n]
        np.testing.assert_array_equal(z.astype(np.uint8), ref_z)
    np.testing.assert_allclose(out["loss"], d["loss"], rtol=1e-5)
    for k in range(int(d["windows"])):
        for g in ("grad_w", "grad_win", "grad_wout", "grad_bout"):
            key = f"{g}_{k}"
            assert rel_err(out[key], d[key]) < 1e-4, (key, rel_err(out[key], d[key]))


@pytest.mark.parametrize("fused", [True, False])
def test_bptt_matches_finite_differences_smooth(fused):
    """Analytic gradient of the smooth-surrogate forward against central
    differences of the same forward (fp32, the 6 largest-gradient weights of
    the recurrent and input layers).  The surrogate backward is
    4 s (1 - s) with s = sigmoid(k alpha u) (sigmoid.py:17-56) whatever the
    forward; with k alpha = 4 it is the exact derivative of the smooth
    forward, so finite differences must agree.  No refractory period: its mask
    (refractory == 0) is a step function of the smooth spike."""
    d = cases.load("train_smooth")
    steps = int(d["steps"])
    k = 2.0 * np.log(np.sqrt(2.0) + 1.0)
    brain, readout, conn, inp = build(d, refractory=False, alpha=4.0 / k, fused=fused)
    x = torch.tensor(d["x"][:steps], device=DEV)
    target = torch.tensor(d["target"][:steps], device=DEV)

    def loss_fn():
        init_net_state(brain, batch_size=int(d["batch"]), dtype=torch.float32, device=DEV)
        with environ.context(dt=1.0):
            z, _ = brain(x)
        return ((readout(z) - target) ** 2).mean()

    loss = loss_fn()
    loss.backward()
    for param in (conn.magnitude, inp.weight):
        g = param.grad.detach().flatten()
        top = torch.topk(g.abs(), 6).indices
        flat = param.data.view(-1)
        for i in top.tolist():
            old = float(flat[i])
            eps = 1e-2 * max(abs(old), 1e-2)
            with torch.no_grad():
                flat[i] = old + eps
                lp = float(loss_fn())
                flat[i] = old - eps
                lm = float(loss_fn())
                flat[i] = old
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - float(g[i])) <= 2e-2 * abs(float(g[i])) + 1e-6, (i, fd, float(g[i]))


def test_fused_bptt_state_stack_gradients_and_alif():
    """Gradients that enter through the returned state stacks (v, psc) and the
    final state, for an ALIF network, equal the per-module path's."""
    import scipy.sparse as sp

    from btorch_b200.models import ALIF

    rng = np.random.default_rng(11)
    n, B, T = 64, 3, 25
    W = sp.random(n, n, density=0.1, random_state=4, dtype=np.float32)
    W.data = (np.round(W.data * 64) / 64 * np.where(rng.random(W.nnz) < 0.8, 1, -1)).astype(np.float32)
    x = torch.tensor((rng.random((T, B, n)) < 0.3).astype(np.float32) * 0.5, device=DEV)
    grads = []
    for fused in (True, False):
        conn = SparseConn(sp.coo_array(W), sparse_config={"direction": "gather"})
        neuron = ALIF(n, v_threshold=1.0, v_reset=0.0, c_m=1.0, g_leak=0.05, E_leak=0.0, E_k=-1.0,
                      tau_adapt=50.0, dg_k=0.1, tau_ref=None, hard_reset=False, surrogate_function=Sigmoid(alpha=3.0))
        brain = RecurrentNN(neuron, ExponentialPSC(n, tau_syn=5.0, linear=conn),
                            update_state_names=("neuron.v", "synapse.psc"), fused=fused).to(DEV)
        init_net_state(brain, batch_size=B, dtype=torch.float32, device=DEV)
        with environ.context(dt=1.0):
            z, st = brain(x)
        assert brain.last_path == ("fused-bptt" if fused else "modular")
        loss = (z * torch.linspace(0.5, 1.5, n, device=DEV)).sum() + (st["neuron.v"] ** 2).mean() \
            + st["synapse.psc"].sum() * 0.1 + brain.neuron.g_k.sum() * 0.3
        loss.backward()
        grads.append(conn.magnitude.grad.cpu().numpy())
    assert rel_err(grads[0], grads[1]) < 1e-5, rel_err(grads[0], grads[1])


def test_fused_bptt_releases_buffers_and_supports_retain_graph():
    """The step buffers are freed with the graph (no reference cycle through
    the module), and a second backward with retain_graph=True gives the same
    gradient again."""
    import gc

    d = cases.load("train_spiking")
    brain, readout, conn, inp = build(d, "gather")
    x = torch.tensor(np.tile(d["x"], (50, 1, 1)), device=DEV)  # 3000 steps: ~30 MB of step buffers
    torch.cuda.synchronize()
    base = torch.cuda.memory_allocated()
    with environ.context(dt=1.0):
        z, st = brain(x)
    assert brain.last_path == "fused-bptt"
    loss = readout(z).square().mean()
    loss.backward(retain_graph=True)
    g1 = conn.magnitude.grad.clone()
    conn.magnitude.grad = None
    loss.backward()
    torch.testing.assert_close(conn.magnitude.grad, g1, rtol=0, atol=0)
    del z, st, loss
    detach_net(brain)
    gc.collect()
    torch.cuda.synchronize()
    held = torch.cuda.memory_allocated() - base
    # the step buffers of this call take ~31 MB; what stays is the gradients
    # and cached packed weights (tens of KB)
    assert held < (8 << 20), held


@pytest.mark.parametrize("kind", ["lif", "alif"])
def test_fused_bptt_checkpointed_recompute_equals_stored_buffers(kind):
    """grad_checkpoint=True: the fused BPTT keeps the state at each chunk start
    and recomputes every chunk in backward.  Spikes, loss, the recurrent,
    input-layer and readout gradients equal those of the run that stores
    every step's buffers (dyadic weights: the recomputation is exact; the
    weight gradients are summed chunk by chunk, so within 1e-6), and the
    buffers take at most a quarter of the stored run's."""
    import scipy.sparse as sp

    from btorch_b200.models import ALIF

    rng = np.random.default_rng(21)
    n, B, T, c_in = 512, 8, 60, 32
    dense = (rng.random((n, n)) < 0.05) * rng.geometric(0.25, (n, n)) * 2.0**-8
    dense[int(0.8 * n):] *= -4.0
    W = sp.coo_array(dense.astype(np.float32))
    w_in = (np.round(rng.normal(0, 0.2, (c_in, n)) * 64) / 64).astype(np.float32)
    x = torch.tensor(rng.poisson(0.2, (T, B, c_in)).astype(np.float32), device=DEV)
    w_out = torch.tensor(rng.normal(0, 0.1, (5, n)).astype(np.float32))
    outs = []
    for ckpt in (False, True):
        conn = SparseConn(W, sparse_config={"direction": "gather"})
        if kind == "lif":
            neuron = LIF(n, tau_ref=2.0, hard_reset=True, surrogate_function=Sigmoid(alpha=5.0))
        else:
            neuron = ALIF(n, g_leak=0.05, E_leak=0.0, E_k=-1.0, tau_adapt=50.0, dg_k=0.0625, tau_ref=2.0,
                          hard_reset=True, surrogate_function=Sigmoid(alpha=5.0))
        inp = DenseConn(c_in, n, weight=torch.tensor(w_in))
        brain = RecurrentNN(neuron, ExponentialPSC(n, tau_syn=5.0, linear=conn), neuron_inp_module=inp,
                            update_state_names=(), grad_checkpoint=ckpt, chunk_size=12, unroll=4).to(DEV)
        readout = torch.nn.Linear(n, 5).to(DEV)
        with torch.no_grad():
            readout.weight.copy_(w_out)
            readout.bias.zero_()
        init_net_state(brain, batch_size=B, dtype=torch.float32, device=DEV)
        with environ.context(dt=1.0):
            z, _ = brain(x)
        assert brain.last_path == "fused-bptt"
        assert brain.last_bptt["recomputed"] == ckpt
        loss = (readout(z) - 0.1).square().mean() + brain.neuron.v.square().mean()
        loss.backward()
        outs.append({"z": z.detach().cpu().numpy(), "loss": float(loss), "w": conn.magnitude.grad.cpu().numpy(),
                     "win": inp.weight.grad.cpu().numpy(), "wout": readout.weight.grad.cpu().numpy(),
                     "bytes": brain.last_bptt["bytes"]})
    a, b = outs
    assert a["z"].sum() > 100
    np.testing.assert_array_equal(a["z"], b["z"])
    assert a["loss"] == b["loss"]
    for key in ("w", "win", "wout"):
        assert rel_err(b[key], a[key]) < 1e-6, (key, rel_err(b[key], a[key]))
    assert b["bytes"] <= 0.35 * a["bytes"]  # T 60, chunks of 12: the spikes are most of what remains
