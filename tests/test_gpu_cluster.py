"""The single-cluster persistent engine (BT_MODE_CLUSTER): every step of a
call in one launch of one thread-block cluster of up to 16 CTAs, the state
and the in-edges in shared memory, ordered in-edge sums, spike words
exchanged through distributed shared memory, one hardware cluster barrier
per step.  Its results are the reference's bit for bit (checked against the
CPU oracle) for any weights, for 1 to 256 samples, LIF and ALIF, with an
input layer, uneven sample lengths, traces, several calls in a row and
CUDA-graph replay, and equal to the gather engine's."""

import numpy as np
import pytest
import torch

from btorch_b200 import _lib as L
from btorch_b200.models import environ
from btorch_b200.models.autotune import EngineChoice
from oracle import oracle as O
from tests.test_gpu_tile import _dyadic, _model, _spec

pytestmark = pytest.mark.gpu
SCATTER = EngineChoice(L.BT_MODE_SCATTER)
GATHER = EngineChoice(L.BT_MODE_GATHER)


def cluster(ctas=0):
    return EngineChoice(L.BT_MODE_CLUSTER, tile_posts=ctas)


@pytest.mark.parametrize("n,batch,ctas", [(2000, 1, 0), (2000, 8, 0), (2000, 33, 0), (1000, 64, 0),
                                          (512, 160, 16), (300, 256, 16), (700, 4, 3), (90, 2, 1),
                                          (1024, 2, 0)])
def test_cluster_lif_bitwise_vs_oracle_uneven_lengths_two_calls(n, batch, ctas):
    rng = np.random.default_rng(200 + batch + n)
    T = 70
    conn = _dyadic(rng, n, min(0.05, 40.0 / n))
    x = (np.round(rng.poisson(0.08, (T, batch, n)) * 0.5 * 64) / 64).astype(np.float32)
    lens = rng.integers(T // 2, T + 10, batch)
    rnn = _model(conn, n, 0, batch)
    spec = _spec(conn, n, 0)
    ost = O.init_state(spec, batch)
    choice = cluster(ctas)
    for a, b in ((0, 30), (30, T)):
        sl = torch.tensor(np.clip(lens - a, 0, b - a), device="cuda")
        with torch.no_grad(), environ.context(dt=1.0):
            z, st = rnn(torch.tensor(x[a:b], device="cuda"), sample_len=sl, engine_choice=choice, engine_stats=True)
        assert rnn.last_engine_choice == choice
        assert rnn.last_engine_launches == 1  # one launch for the whole call
        o = O.run(spec, ost, x[a:b], sample_len=np.clip(lens - a, 0, b - a).astype(np.int32), want_v=True,
                  want_psc=True, events=True)
        np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), o["spikes"])
        np.testing.assert_array_equal(st["neuron.v"].cpu().numpy(), o["v"])
        np.testing.assert_array_equal(st["synapse.psc"].cpu().numpy(), o["psc"])
        outdeg = np.bincount(conn.tocoo().row, minlength=n)
        events = (o["spikes"].astype(np.int64) * outdeg[None, None, :]).sum(axis=(1, 2))
        np.testing.assert_array_equal(rnn.last_engine_stats[:, 1].cpu().numpy(), events)
        union = o["spikes"].any(axis=1).sum(axis=1)
        np.testing.assert_array_equal(rnn.last_engine_stats[:, 0].cpu().numpy(), union)
    assert o["spikes"].sum() > 20
    np.testing.assert_array_equal(rnn.neuron.v.cpu().numpy(), ost.v)
    np.testing.assert_array_equal(rnn.synapse.psc.cpu().numpy(), ost.psc)


@pytest.mark.parametrize("n,batch", [(4096, 1), (1500, 5)])
def test_cluster_any_weights_bitwise_vs_oracle_and_gather(n, batch):
    """Non-dyadic weights: the in-edge sums run in ascending order like the
    reference's, so the result is still the oracle's (and the gather
    engine's) bit for bit."""
    import scipy.sparse as sp

    rng = np.random.default_rng(31 + n)
    T = 120
    dense = (rng.random((n, n)) < 0.02) * rng.normal(0.0, 0.12, (n, n))
    conn = sp.coo_array(dense.astype(np.float32))
    x = (rng.random((T, batch, n)) < 0.01).astype(np.float32) * rng.normal(1.0, 0.3, (T, batch, n)).astype(np.float32)
    spec = _spec(conn, n, 0)
    o = O.run(spec, O.init_state(spec, batch), x, want_v=True, want_psc=True, events=True)
    outs = []
    for choice in (cluster(), GATHER):
        rnn = _model(conn, n, 0, batch)
        with torch.no_grad(), environ.context(dt=1.0):
            z, st = rnn(torch.tensor(x, device="cuda"), engine_choice=choice)
        outs.append((z.cpu().numpy(), st["neuron.v"].cpu().numpy(), st["synapse.psc"].cpu().numpy()))
    assert o["spikes"].sum() > 200
    np.testing.assert_array_equal(outs[0][0].astype(np.uint8), o["spikes"])
    np.testing.assert_array_equal(outs[0][1], o["v"])
    np.testing.assert_array_equal(outs[0][2], o["psc"])
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def test_cluster_shape_and_too_large_network():
    from btorch_b200.models.engine import cluster_shape

    sl_ptr = np.arange(0, 129) * 64  # 128 slices of 64 rows: n = 4096
    assert cluster_shape(4096, 1, sl_ptr) == (256, 16, 512)
    assert cluster_shape(4096, 1, sl_ptr, ctas=8) == (512, 8, 1024)
    assert cluster_shape(4096, 1, np.arange(0, 129) * 61) == (256, 16, 512)  # slices rounded up to 64 rows
    assert cluster_shape(4096, 1, sl_ptr * 2, ctas=8) is None  # 1920 rows: 368 KB of edges
    assert cluster_shape(4096, 1, np.arange(0, 129) * 1000) is None  # 8000 rows a tile
    import scipy.sparse as sp

    n = 8192  # in-degree ~200: about 700 KB of in-edges a tile
    conn = sp.random(n, n, density=0.025, format="coo", dtype=np.float32, random_state=1)
    conn.data[:] = 2.0**-8
    rnn = _model(conn, n, 0, 1)
    with pytest.raises(NotImplementedError, match="cluster"):
        with torch.no_grad(), environ.context(dt=1.0):
            rnn(torch.zeros(4, 1, n, device="cuda"), engine_choice=cluster())


@pytest.mark.parametrize("batch", [3, 32])
def test_cluster_alif_with_input_layer_equals_scatter_step(batch):
    """ALIF + dense input layer: cluster == two-launch scatter, bit for bit
    (dyadic weights and input): rasters, traces and final state."""
    rng = np.random.default_rng(17 + batch)
    n, T, c_in = 3000, 60, 40
    conn = _dyadic(rng, n, 0.01, exp=-6)
    w_in = (np.round(rng.normal(0, 0.3, (c_in, n)) * 64) / 64).astype(np.float32)
    x = torch.tensor(rng.poisson(0.1, (T, batch, c_in)).astype(np.float32), device="cuda")
    outs = []
    for choice in (SCATTER, cluster(), GATHER):
        rnn = _model(conn, n, 1, batch, c_in, w_in, names=("neuron.v", "neuron.g_k", "synapse.psc"))
        with torch.no_grad(), environ.context(dt=1.0):
            z, st = rnn(x, engine_choice=choice)
        outs.append([z.cpu().numpy(), st["neuron.v"].cpu().numpy(), st["neuron.g_k"].cpu().numpy(),
                     st["synapse.psc"].cpu().numpy(), rnn.neuron.v.cpu().numpy(), rnn.synapse.psc.cpu().numpy()])
    assert outs[0][0].sum() > 100
    for other in outs[1:]:
        for a, b in zip(outs[0], other):
            np.testing.assert_array_equal(a, b)


def test_cluster_graph_replay_equals_eager_and_bitmask_output():
    rng = np.random.default_rng(4)
    n, T, B = 4096, 300, 1
    conn = _dyadic(rng, n, 0.02)
    x = torch.tensor((np.round(rng.poisson(0.03, (T, B, n)) * 0.5 * 64) / 64).astype(np.float32), device="cuda")
    outs = []
    for graph in (False, True):
        rnn = _model(conn, n, 0, B, names=())
        rnn.cudagraph = graph
        with torch.no_grad(), environ.context(dt=1.0):
            r1, _ = rnn(x, spikes_out="bitmask", engine_choice=cluster())
            r2, _ = rnn(x, spikes_out="bitmask", engine_choice=cluster())
        outs.append((r1.cpu().numpy(), r2.cpu().numpy(), rnn.neuron.v.cpu().numpy()))
    assert outs[0][0].any()
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def test_cluster_wait_timeout_is_reported_and_the_context_stays_usable():
    """A spike-word wait limited to one poll gives up: every CTA stops waiting
    and publishing, the launch ends, the call raises, and the next call
    (default limit) is correct again."""
    rng = np.random.default_rng(6)
    n, T, B = 4096, 100, 1
    conn = _dyadic(rng, n, 0.02)
    x = (np.round(rng.poisson(0.05, (T, B, n)) * 0.5 * 64) / 64).astype(np.float32)
    rnn = _model(conn, n, 0, B, names=())
    rnn.engine_spin_limit = 1
    with pytest.raises(RuntimeError, match="gave up"):
        with torch.no_grad(), environ.context(dt=1.0):
            rnn(torch.tensor(x, device="cuda"), engine_choice=cluster())
    torch.cuda.synchronize()
    rnn.engine_spin_limit = 0
    from btorch_b200.models.functional import init_net_state

    init_net_state(rnn, batch_size=B, dtype=torch.float32, device="cuda")
    with torch.no_grad(), environ.context(dt=1.0):
        z, _ = rnn(torch.tensor(x, device="cuda"), engine_choice=cluster())
    spec = _spec(conn, n, 0)
    o = O.run(spec, O.init_state(spec, B), x, events=True)
    np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), o["spikes"])


def test_cluster_deferred_status_reports_at_engine_status():
    """engine_status_check = "deferred": the call that gave up returns
    without a host synchronisation; engine_status() raises for it."""
    rng = np.random.default_rng(8)
    n, T, B = 4096, 100, 1
    conn = _dyadic(rng, n, 0.02)
    x = torch.tensor((np.round(rng.poisson(0.05, (T, B, n)) * 0.5 * 64) / 64).astype(np.float32), device="cuda")
    rnn = _model(conn, n, 0, B, names=())
    rnn.engine_status_check = "deferred"
    rnn.engine_spin_limit = 1
    with torch.no_grad(), environ.context(dt=1.0):
        rnn(x, engine_choice=cluster())
    with pytest.raises(RuntimeError, match="gave up"):
        rnn.engine_status()
    rnn.engine_spin_limit = 0
    with torch.no_grad(), environ.context(dt=1.0):
        rnn(x, engine_choice=cluster())
    rnn.engine_status()  # nothing pending that failed


# ------------------------------------------------------------ delay bins --

@pytest.mark.parametrize("name", ["delayed_psc", "hetero_delay", "lif_dyadic_soft", "lif_dyadic_input"])
def test_cluster_bitwise_vs_reference_fixtures(name):
    """The reference's own runs (golden fixtures; DelayedPSC's uniform delay,
    HeterSynapsePSC's per-synapse delay bins, no delays): spike rasters, v
    and psc traces and the final state bit for bit, in one launch."""
    from tests import cases

    d = cases.load(name)
    rnn, psc_name = cases.build_model(d, "cuda", "gather")
    with torch.no_grad(), environ.context(dt=float(d["dt"])):
        z, st = rnn(torch.tensor(d["x"], device="cuda"), engine_choice=cluster())
    assert rnn.last_engine_choice == cluster()
    assert rnn.last_engine_launches == (3 if rnn.neuron_inp_module is not None else 1)  # (+ the projection's 2)
    K = d["v"].shape[0]
    np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), cases.spikes(d))
    np.testing.assert_array_equal(st["neuron.v"].cpu().numpy()[:K].reshape(d["v"].shape), d["v"])
    np.testing.assert_array_equal(st[psc_name].cpu().numpy()[:K].reshape(d["psc"].shape), d["psc"])
    np.testing.assert_array_equal(rnn.neuron.v.cpu().numpy().reshape(d["v_final"].shape), d["v_final"])


@pytest.mark.parametrize("name", ["delayed_psc", "hetero_delay"])
def test_cluster_delays_split_calls_and_uneven_lengths_equal_gather(name):
    """Calls split at several points (the delay history carried across calls
    through the modules), per-sample lengths, graph replay: the cluster engine
    equals the gather engine bit for bit."""
    from tests import cases

    d = cases.load(name)
    x = torch.tensor(d["x"], device="cuda")
    B = x.shape[1]
    lens = torch.tensor([x.shape[0] - 7 * b for b in range(B)], device="cuda")
    outs = []
    for choice in (GATHER, cluster()):
        for graph in (False, True):
            rnn, psc_name = cases.build_model(d, "cuda", "gather")
            rnn.cudagraph = graph
            zs = []
            with torch.no_grad(), environ.context(dt=float(d["dt"])):
                for a, b in ((0, 5), (5, 37), (37, x.shape[0])):
                    z, _ = rnn(x[a:b], sample_len=(lens - a).clamp(min=0, max=b - a), engine_choice=choice)
                    zs.append(z.cpu().numpy())
            outs.append((np.concatenate(zs), rnn.neuron.v.cpu().numpy(), getattr(rnn.synapse, "psc", None)))
    ref = outs[0]
    assert ref[0].sum() > 50
    for o in outs[1:]:
        np.testing.assert_array_equal(o[0], ref[0])
        np.testing.assert_array_equal(o[1], ref[1])


def test_cluster_many_delay_bins_any_weights_equal_gather():
    """A random network with per-synapse delays of 1..12 steps (12 bins, 13
    bitmap copies) and non-dyadic weights, batch 3: the cluster engine's
    ordered sums equal the gather engine's bit for bit over 200 steps."""
    import pandas as pd
    import scipy.sparse as sp

    from btorch_b200.models import LIF, HeterSynapsePSC, RecurrentNN, SparseConn
    from btorch_b200.models.functional import init_net_state

    rng = np.random.default_rng(12)
    n, R, B, T = 1200, 12, 3, 200
    nnz = 40 * n
    pre = rng.integers(0, n, nnz)
    post = rng.integers(0, n, nnz)
    binv = rng.integers(0, R, nnz)
    w = (rng.normal(0.0, 0.25, nnz) * np.where(pre < 0.8 * n, 1.0, -2.0)).astype(np.float32)
    m = sp.coo_array((w, (pre * R + binv, post)), shape=(n * R, n)).tocsr().tocoo()
    x = torch.tensor((rng.random((T, B, n)) < 0.02).astype(np.float32) * 1.5, device="cuda")
    outs = []
    for choice in (GATHER, cluster()):
        rti = pd.DataFrame({"receptor_type": ["syn"], "receptor_index": [0]})
        conn = SparseConn(m, sparse_config={"direction": "gather"})
        syn = HeterSynapsePSC(n, 1, rti, conn, max_delay_steps=R, use_circular_buffer=True, tau_syn=5.0)
        rnn = RecurrentNN(LIF(n, tau_ref=2.0, hard_reset=True), syn, update_state_names=("neuron.v",)).cuda()
        init_net_state(rnn, batch_size=B, dtype=torch.float32, device="cuda")
        with torch.no_grad(), environ.context(dt=1.0):
            z, st = rnn(x, engine_choice=choice)
        outs.append((z.cpu().numpy(), st["neuron.v"].cpu().numpy()))
    assert outs[0][0].sum() > 500
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def test_cluster_repacks_after_a_weight_change():
    """The packed in-edges are reused across calls while the connection's
    parameters are unchanged, and packed again after an in-place change of
    the magnitudes: the run then equals a fresh model with the new weights."""
    rng = np.random.default_rng(21)
    n, T, B = 2000, 40, 2
    conn = _dyadic(rng, n, 0.02)
    x = torch.tensor((np.round(rng.poisson(0.08, (T, B, n)) * 0.5 * 64) / 64).astype(np.float32), device="cuda")
    rnn = _model(conn, n, 0, B, names=())
    with torch.no_grad(), environ.context(dt=1.0):
        rnn(x, engine_choice=cluster())
        packed = rnn.synapse.linear._cluster_packed
        rnn(x, engine_choice=cluster())
        assert rnn.synapse.linear._cluster_packed is packed  # reused
        rnn.synapse.linear.magnitude.mul_(2.0)
        from btorch_b200.models.functional import init_net_state

        init_net_state(rnn, batch_size=B, dtype=torch.float32, device="cuda")
        z, _ = rnn(x, engine_choice=cluster())
    assert rnn.synapse.linear._cluster_packed is not packed
    conn2 = conn.copy()
    conn2.data = conn2.data * 2.0
    fresh = _model(conn2, n, 0, B, names=())
    with torch.no_grad(), environ.context(dt=1.0):
        z2, _ = fresh(x, engine_choice=GATHER)
    np.testing.assert_array_equal(z.cpu().numpy(), z2.cpu().numpy())
    assert z.cpu().numpy().sum() > 50
