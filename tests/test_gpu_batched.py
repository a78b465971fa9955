"""Batched engine runs (mask words 2 and 4, split warps above 128 samples, ALIF,
delays) against the CPU oracle, bit for bit on dyadic weights."""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from btorch_b200.connectome import expand_conn_for_delays
from btorch_b200.models import ALIF, LIF, ExponentialPSC, HeterSynapsePSC, RecurrentNN, SparseConn, environ
from btorch_b200.models._ops import exp_euler_coef
from btorch_b200.models.functional import init_net_state
from oracle import oracle as O

pytestmark = pytest.mark.gpu
MODES = {"gather": {"direction": "gather", "pull_min_batch": 1 << 30},
         "pull": {"direction": "gather", "pull_min_batch": 1},
         "scatter": {"direction": "scatter"}}


def _dyadic_net(rng, n, p, D=1):
    dense = (rng.random((n, n)) < p) * rng.geometric(0.25, (n, n)) * 2.0**-7
    dense[int(0.8 * n):] *= -1.0
    base = sp.coo_array(dense.astype(np.float32))
    if D > 1:
        return expand_conn_for_delays(base, rng.integers(0, D, size=base.nnz), n_delay_bins=D)
    return base


def _oracle_spec(conn, n, kind, D, dt=1.0):
    c = conn.tocoo().T
    c.sum_duplicates()
    ptr = np.concatenate([[0], np.cumsum(np.bincount(c.row, minlength=n))]).astype(np.int64)
    coef = float(exp_euler_coef(torch.tensor(5.0), dt)[0])
    P = {"v_threshold": 1.0, "v_reset": 0.0, "c_m": 1.0, "tau_ref": 2.0, "psc_coef": coef, "psc_tau": 5.0}
    if kind == 0:
        P["tau"] = 20.0
    else:
        P.update(g_leak=0.05, E_leak=0.0, E_k=-1.0, dg_k=0.0625, tau_adapt=200.0,
                 coef_gk=float(exp_euler_coef(torch.tensor(200.0), dt)[0]))
    return O.NetSpec(n=n, kind=kind, hard_reset=True, use_ref=True, dt=dt, params=P, ptr=ptr,
                     pre=(c.col // D).astype(np.int32), delay=(c.col % D).astype(np.int32),
                     w=c.data.astype(np.float32), max_delay=D - 1)


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("batch", [40, 100, 160])
def test_batched_lif_bitwise_vs_oracle(batch, mode):
    rng = np.random.default_rng(batch)
    n, T = 300, 60
    conn = _dyadic_net(rng, n, 0.05)
    x = (np.round(rng.poisson(0.08, (T, batch, n)) * 0.5 * 64) / 64).astype(np.float32)
    rnn = RecurrentNN(LIF(n, tau_ref=2.0, hard_reset=True),
                      ExponentialPSC(n, 5.0, SparseConn(conn, sparse_config=MODES[mode])),
                      update_state_names=("neuron.v",)).cuda()
    init_net_state(rnn, batch_size=batch, dtype=torch.float32, device="cuda")
    with torch.no_grad(), environ.context(dt=1.0):
        z, st = rnn(torch.tensor(x, device="cuda"), engine_stats=True)
    spec = _oracle_spec(conn, n, 0, 1)
    ost = O.init_state(spec, batch)
    o = O.run(spec, ost, x, want_v=True)
    np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), o["spikes"])
    np.testing.assert_array_equal(st["neuron.v"].cpu().numpy(), o["v"])
    # per-step event statistics agree with the raster
    outdeg = np.bincount(conn.tocoo().row, minlength=n)
    events = (o["spikes"].astype(np.int64) * outdeg[None, None, :]).sum(axis=(1, 2))
    np.testing.assert_array_equal(rnn.last_engine_stats[:, 1].cpu().numpy(), events)


@pytest.mark.parametrize("mode", sorted(MODES))
def test_batched_alif_delays_vs_oracle(mode):
    rng = np.random.default_rng(5)
    n, T, B, D = 256, 50, 70, 4
    conn = _dyadic_net(rng, n, 0.05, D)
    x = (np.round(rng.poisson(0.08, (T, B, n)) * 0.75 * 64) / 64).astype(np.float32)
    import pandas as pd

    rti = pd.DataFrame({"receptor_type": ["a"], "receptor_index": [0]})
    syn = HeterSynapsePSC(n, 1, rti, SparseConn(conn, sparse_config=MODES[mode]), base_psc=ExponentialPSC,
                          max_delay_steps=D, use_circular_buffer=True, tau_syn=5.0)
    neuron = ALIF(n, g_leak=0.05, E_leak=0.0, E_k=-1.0, dg_k=0.0625, tau_adapt=200.0, tau_ref=2.0, hard_reset=True)
    rnn = RecurrentNN(neuron, syn, update_state_names=("neuron.v",)).cuda()
    init_net_state(rnn, batch_size=B, dtype=torch.float32, device="cuda")
    with torch.no_grad(), environ.context(dt=1.0):
        z, st = rnn(torch.tensor(x, device="cuda"))
    spec = _oracle_spec(conn, n, 1, D)
    ost = O.init_state(spec, B)
    o = O.run(spec, ost, x, want_v=True)
    zz = z.cpu().numpy().astype(np.uint8)
    bad = np.nonzero((zz != o["spikes"]).reshape(T, -1).any(1))[0]
    k = int(bad[0]) if bad.size else T
    assert k >= 20, f"spikes diverged at step {k}"
    np.testing.assert_allclose(st["neuron.v"].cpu().numpy()[:k], o["v"][:k], rtol=1e-5, atol=1e-5)
