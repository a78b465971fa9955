"""Rows beyond the core step, against the reference's own outputs:
SparseConstrainedConn (grouped magnitudes) forward and backward, and
HeterSynapsePSC with two receptors (per-receptor time constants) in a
recurrent run."""

import numpy as np
import pandas as pd
import pytest
import scipy.sparse as sp
import torch

from btorch_b200.models import LIF, ExponentialPSC, HeterSynapsePSC, RecurrentNN, SparseConn, SparseConstrainedConn
from btorch_b200.models import environ
from btorch_b200.models.functional import init_net_state
from tests import cases

pytestmark = pytest.mark.gpu
DEV = "cuda"


def constrained(d, direction):
    C = sp.coo_array((d["C_data"], (d["C_row"], d["C_col"])), shape=d["W"].shape)
    m = SparseConstrainedConn(sp.coo_array(d["W"]), C, sparse_config={"direction": direction}).to(DEV)
    with torch.no_grad():
        m.magnitude.copy_(torch.tensor(d["magnitude"]))
    return m


@pytest.mark.parametrize("direction", ["gather", "scatter"])
def test_constrained_conn_matches_reference(direction):
    d = cases.load("constrained_spmm")
    m = constrained(d, direction)
    np.testing.assert_array_equal(m._constraint_scatter_indices.cpu().numpy(), d["group"])
    x = torch.tensor(d["x"], device=DEV, requires_grad=True)
    out = m(x)
    (out * torch.tensor(d["g"], device=DEV)).sum().backward()
    if direction == "gather":
        np.testing.assert_array_equal(out.detach().cpu().numpy(), d["out"])
    else:
        np.testing.assert_allclose(out.detach().cpu().numpy(), d["out"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(x.grad.cpu().numpy(), d["grad_x"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(m.magnitude.grad.cpu().numpy(), d["grad_mag"], rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("direction", ["gather", "scatter"])
def test_two_receptor_hetersynapse_matches_reference(direction):
    d = cases.load("receptors2")
    n, R = int(d["n"]), int(d["n_rec"])
    W = sp.coo_array((d["w"], (d["src"], d["post"])), shape=(n, n * R))
    conn = SparseConn(W, sparse_config={"direction": direction})
    rti = pd.DataFrame({"receptor_type": [f"r{r}" for r in range(R)], "receptor_index": list(range(R))})
    syn = HeterSynapsePSC(n, R, rti, conn, base_psc=ExponentialPSC, tau_syn=torch.tensor(np.tile(d["taus"], n)))
    rnn = RecurrentNN(LIF(n, tau_ref=2.0, hard_reset=True), syn,
                      update_state_names=("neuron.v", "synapse.psc", "synapse.base_psc.psc")).to(DEV)
    init_net_state(rnn, batch_size=int(d["batch"]), dtype=torch.float32, device=DEV)
    with torch.no_grad(), environ.context(dt=1.0):
        z, st = rnn(torch.tensor(d["x"], device=DEV))
    assert rnn.last_path == "fused" and rnn.last_engine_direction == direction
    ref_z = np.unpackbits(d["z"], axis=-1, bitorder="little")[..., :n]
    np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), ref_z)
    K = d["v"].shape[0]
    np.testing.assert_array_equal(st["neuron.v"].cpu().numpy()[:K], d["v"])
    np.testing.assert_array_equal(st["synapse.psc"].cpu().numpy()[:K], d["psc"])
    np.testing.assert_array_equal(st["synapse.base_psc.psc"].cpu().numpy()[:K], d["psc_rec"])


@pytest.mark.parametrize("direction", ["gather", "scatter"])
def test_empty_connection_equals_zero_weight_network(direction):
    """A connection without synapses (valid in the reference: torch.sparse.mm
    of an empty matrix) runs on the per-module kernels and gives the same
    rasters, states and input gradients as the same network with one
    zero-weight synapse on the fused paths; its weight gradient is empty."""
    n, B, T = 64, 3, 40
    rng = np.random.default_rng(5)
    x = torch.tensor((rng.poisson(0.3, (T, B, n)) * 0.75).astype(np.float32), device=DEV)
    r = torch.tensor(rng.standard_normal((T, B, n)).astype(np.float32), device=DEV)

    def model(mat):
        conn = SparseConn(mat, sparse_config={"direction": direction})
        rnn = RecurrentNN(LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True),
                          ExponentialPSC(n, tau_syn=5.0, linear=conn)).to(DEV)
        init_net_state(rnn, batch_size=B, dtype=torch.float32, device=DEV)
        return rnn, conn

    empty, c_empty = model(sp.coo_array((n, n), dtype=np.float32))
    zero, _ = model(sp.coo_array((np.zeros(1, np.float32), ([0], [1])), shape=(n, n)))
    with torch.no_grad(), environ.context(dt=1.0):
        z0, s0 = empty(x)
        z1, s1 = zero(x)
    assert empty.last_path == "modular" and zero.last_path == "fused"
    assert torch.equal(z0, z1) and z0.sum() > 0
    assert s0.keys() == s1.keys()
    for k in s0:
        assert torch.equal(s0[k], s1[k]), k

    grads = []
    for rnn in (empty, zero):
        init_net_state(rnn, batch_size=B, dtype=torch.float32, device=DEV)
        xg = x.clone().requires_grad_(True)
        with environ.context(dt=1.0):
            z, _ = rnn(xg)
        (z * r).sum().backward()
        grads.append(xg.grad)
    assert empty.last_path == "modular" and zero.last_path == "fused-bptt"
    assert grads[0].abs().sum() > 0
    # fused BPTT and per-module backward: same chain, summed in its own order
    assert (grads[0] - grads[1]).norm() <= 1e-5 * grads[1].norm()
    assert c_empty.magnitude.grad is not None and c_empty.magnitude.grad.shape == (0,)
