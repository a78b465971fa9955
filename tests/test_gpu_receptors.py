"""Receptor channels end to end: a connectome table -> make_hetersynapse_conn
(E/I neuron mode, 4 receptor pairs, per-synapse delays over 5 bins) ->
HeterSynapsePSC(n_receptor=4, ExponentialPSC with a time constant per
receptor) -> RecurrentNN, against the reference's own run of the same tables
(tests/golden/receptors_delay.npz): spike raster, v, receptor-summed psc and
the per-channel base psc bit for bit, through the fused engine (gather and
scatter, eager and CUDA graph) and the per-module path."""

import numpy as np
import pandas as pd
import pytest
import scipy.sparse as sp
import torch

from btorch_b200.connectome import make_hetersynapse_conn
from btorch_b200.models import LIF, ExponentialPSC, HeterSynapsePSC, RecurrentNN, SparseConn, environ
from btorch_b200.models.functional import init_net_state
from tests import cases

pytestmark = pytest.mark.gpu
DEV = "cuda"


def build(d, direction):
    n, D = int(d["n"]), int(d["n_bins"])
    neu = pd.DataFrame({k.split(".", 1)[1]: v for k, v in d.items() if k.startswith("neurons.")})
    con = pd.DataFrame({k.split(".", 1)[1]: v for k, v in d.items() if k.startswith("conns.")})
    neu["EI"] = neu["EI"].astype(object)
    m, idx = make_hetersynapse_conn(neu, con, delay_col="delay_steps", n_delay_bins=D)
    m = m.tocoo()
    inh = (neu.EI.to_numpy() == "I")[m.row // D]
    w = (m.data * 2.0**-5 * np.where(inh, -1.0, 1.0)).astype(np.float32)
    conn = SparseConn(sp.coo_array((w, (m.row, m.col)), shape=m.shape), sparse_config={"direction": direction})
    # the connection is the reference's, entry for entry (canonical order)
    np.testing.assert_array_equal(conn.indices[0].numpy(), d["post"])
    np.testing.assert_array_equal(conn.indices[1].numpy(), d["src"])
    C = len(idx)
    syn = HeterSynapsePSC(n, C, idx, conn, base_psc=ExponentialPSC, max_delay_steps=D, use_circular_buffer=True,
                          tau_syn=torch.tensor(np.tile(d["taus"], n)))
    rnn = RecurrentNN(LIF(n, tau_ref=2.0, hard_reset=True), syn,
                      update_state_names=("neuron.v", "synapse.psc", "synapse.base_psc.psc")).to(DEV)
    init_net_state(rnn, batch_size=int(d["batch"]), dtype=torch.float32, device=DEV)
    return rnn


@pytest.mark.parametrize("path", ["gather", "scatter", "gather-graph", "scatter-graph", "modular"])
def test_receptors_with_delays_match_reference(path):
    d = cases.load("receptors_delay")
    n = int(d["n"])
    direction = path.split("-")[0] if path != "modular" else "gather"
    rnn = build(d, direction)
    rnn.fused = path != "modular"
    rnn.cudagraph = path.endswith("graph")
    x = torch.tensor(d["x"], device=DEV)
    with torch.no_grad(), environ.context(dt=1.0):
        if rnn.cudagraph:
            z1, st1 = rnn(x[:48], engine_chunk=12)
            z2, st2 = rnn(x[48:], engine_chunk=12)
            z = torch.cat([z1, z2])
            st = {k: torch.cat([st1[k], st2[k]]) for k in st1}
        else:
            z, st = rnn(x)
    assert rnn.last_path == ("modular" if path == "modular" else "fused")
    if path != "modular":
        assert rnn.last_engine_direction == direction
    np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), cases.spikes(d))
    K = d["v"].shape[0]
    np.testing.assert_array_equal(st["neuron.v"].cpu().numpy()[:K], d["v"])
    np.testing.assert_array_equal(st["synapse.psc"].cpu().numpy()[:K], d["psc"])
    np.testing.assert_array_equal(st["synapse.base_psc.psc"].cpu().numpy()[:K], d["psc_rec"])
    np.testing.assert_array_equal(rnn.neuron.v.cpu().numpy(), d["v_final"])
    np.testing.assert_array_equal(rnn.synapse.psc.cpu().numpy(), d["psc_final"])
    np.testing.assert_array_equal(rnn.synapse.base_psc.psc.cpu().numpy(), d["psc_rec_final"])
    # receptor channel lookup (synapse.py:763-830)
    ee = rnn.synapse.get_psc(("E", "E"))
    assert ee.shape == (int(d["batch"]), n)
    np.testing.assert_array_equal(ee.cpu().numpy(), d["psc_rec_final"].reshape(-1, n, 4)[..., 0])


def test_receptor_sum_order_on_gpu():
    """The GPU receptor sum replays torch's CPU order: equal to torch.sum on
    the CPU for 1..16 channels on values whose sums round differently in
    other orders."""
    from btorch_b200.models.synapse import receptor_sum

    rng = np.random.default_rng(5)
    for C in range(1, 17):
        a = (rng.standard_normal((64, 300, C)) * np.exp(rng.standard_normal((64, 300, C)) * 3)).astype(np.float32)
        t = torch.tensor(a)
        np.testing.assert_array_equal(receptor_sum(t.to(DEV)).cpu().numpy(), t.sum(-1).numpy(), err_msg=str(C))


def test_inplace_reset_after_inference_run():
    """A fused run under inference_mode leaves the modules' state tensors
    usable by an in-place reset outside it (the serving / benchmark loop)."""
    from btorch_b200.models.functional import reset_net

    d = cases.load("receptors_delay")
    rnn = build(d, "scatter")
    rnn.update_state_names = ()
    x = torch.tensor(d["x"], device=DEV)
    for _ in range(2):
        reset_net(rnn, inplace=True)
        with torch.inference_mode(), environ.context(dt=1.0):
            z, _ = rnn(x)
        np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), cases.spikes(d))


@pytest.mark.parametrize("direction", ["gather", "scatter"])
def test_host_streamed_receptor_run_with_traces(direction):
    """A host-resident input streamed through the fused receptor engine, with
    every state trace requested (per-channel psc, summed psc, v) and uneven
    sample lengths: identical to the device-input run, outputs on the host."""
    d = cases.load("receptors_delay")
    x = torch.tensor(d["x"])
    lens = torch.tensor([120, 33, 80][: int(d["batch"])])
    outs = []
    for host in (False, True):
        rnn = build(d, direction)
        xin = x.pin_memory() if host else x.to(DEV)
        with torch.no_grad(), environ.context(dt=1.0):
            z, st = rnn(xin, sample_len=lens, engine_chunk=40)
        assert z.device.type == ("cpu" if host else "cuda")
        outs.append([z.cpu().numpy()] + [st[k].cpu().numpy() for k in sorted(st)] +
                    [rnn.synapse.base_psc.psc.cpu().numpy(), rnn.neuron.v.cpu().numpy()])
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("direction", ["gather", "scatter"])
@pytest.mark.parametrize("C", [3, 9])
def test_odd_receptor_counts_match_oracle(C, direction):
    """Receptor counts without a vector path (3) and with the eight-accumulator
    sum (9, the E/I/unknown pairs): the fused engine against the oracle, bit
    for bit (dyadic weights, per-synapse delays over 4 bins)."""
    from oracle import oracle as O

    rng = np.random.default_rng(C)
    n, B, T, D = 200, 3, 90, 4
    nnz = 3000
    post = rng.integers(0, n * C, nnz)
    src = rng.integers(0, n * D, nnz)
    key = np.unique(post * (n * D) + src)
    post, src = key // (n * D), key % (n * D)
    w = (rng.integers(1, 6, key.size) * np.where(rng.random(key.size) < 0.8, 1.0, -1.0) * 2.0 ** -4).astype(np.float32)
    taus = np.tile((2.0 + rng.integers(0, 8, C)).astype(np.float32), n)
    x = (np.round(rng.poisson(0.1, (T, B, n)) * 0.75 * 64) / 64).astype(np.float32)
    conn = SparseConn(sp.coo_array((w, (src, post)), shape=(n * D, n * C)), sparse_config={"direction": direction})
    rti = pd.DataFrame({"receptor_type": [f"r{r}" for r in range(C)], "receptor_index": list(range(C))})
    syn = HeterSynapsePSC(n, C, rti, conn, base_psc=ExponentialPSC, max_delay_steps=D, use_circular_buffer=True,
                          tau_syn=torch.tensor(taus))
    rnn = RecurrentNN(LIF(n, tau_ref=2.0, hard_reset=True), syn, update_state_names=("neuron.v",)).to(DEV)
    init_net_state(rnn, batch_size=B, dtype=torch.float32, device=DEV)
    with torch.no_grad(), environ.context(dt=1.0):
        z, st = rnn(torch.tensor(x, device=DEV))
    assert rnn.last_path == "fused" and rnn.last_engine_direction == direction
    ptr = np.concatenate([[0], np.cumsum(np.bincount(post, minlength=n * C))]).astype(np.int64)
    coef = syn.base_psc.coefficients(1.0)[0].cpu().numpy()
    spec = O.NetSpec(n=n, kind=0, hard_reset=True, use_ref=True, dt=1.0,
                     params={"v_threshold": 1.0, "v_reset": 0.0, "c_m": 1.0, "tau": 20.0, "tau_ref": 2.0,
                             "psc_coef": coef, "psc_tau": taus},
                     ptr=ptr, pre=(src // D).astype(np.int32), delay=(src % D).astype(np.int32), w=w,
                     max_delay=D - 1, n_rec=C)
    ost = O.init_state(spec, B)
    o = O.run(spec, ost, x, want_v=True, threads=4)
    np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), o["spikes"])
    np.testing.assert_array_equal(st["neuron.v"].cpu().numpy(), o["v"])
    np.testing.assert_array_equal(rnn.synapse.base_psc.psc.cpu().numpy(), ost.psc)
