"""The persistent tile engine (BT_MODE_TILE): many steps per launch, one CTA
per tile of posts with the tile's synaptic input in shared memory, a bounded
grid barrier per step.  On dyadic weights its results are the reference's bit
for bit (checked against the CPU oracle), for every mask width (batches 1 to
160), LIF and ALIF, with an input layer, uneven sample lengths, state
traces, several calls in a row, CUDA-graph replay, and against the
two-launch scatter step.  A barrier whose wait is made to give up ends the
launch with BT_ERR_TIMEOUT, reported on the host, and the context stays
usable."""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from btorch_b200 import _lib as L
from btorch_b200.models import ALIF, LIF, DenseConn, ExponentialPSC, RecurrentNN, SparseConn, environ
from btorch_b200.models._ops import exp_euler_coef
from btorch_b200.models.autotune import EngineChoice
from btorch_b200.models.functional import init_net_state
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TILE = EngineChoice(L.BT_MODE_TILE)
SCATTER = EngineChoice(L.BT_MODE_SCATTER)


def _dyadic(rng, n, p, exp=-7):
    dense = (rng.random((n, n)) < p) * rng.geometric(0.25, (n, n)) * 2.0**exp
    dense[int(0.8 * n):] *= -1.0
    return sp.coo_array(dense.astype(np.float32))


def _model(conn, n, kind, batch, c_in=0, w_in=None, names=("neuron.v", "synapse.psc")):
    if kind == 0:
        neuron = LIF(n, tau_ref=2.0, hard_reset=True)
    else:
        neuron = ALIF(n, g_leak=0.05, E_leak=0.0, E_k=-1.0, dg_k=0.0625, tau_adapt=200.0, tau_ref=2.0,
                      hard_reset=True)
    inp = DenseConn(c_in, n, weight=torch.tensor(w_in)) if c_in else None
    rnn = RecurrentNN(neuron, ExponentialPSC(n, 5.0, SparseConn(conn, sparse_config={"direction": "scatter"})),
                      neuron_inp_module=inp, update_state_names=names).cuda()
    init_net_state(rnn, batch_size=batch, dtype=torch.float32, device="cuda")
    return rnn


def _spec(conn, n, kind, dt=1.0):
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
                     pre=c.col.astype(np.int32), delay=np.zeros(c.nnz, np.int32), w=c.data.astype(np.float32))


@pytest.mark.parametrize("batch", [1, 8, 40, 100, 160])
def test_tile_lif_bitwise_vs_oracle_uneven_lengths_two_calls(batch):
    rng = np.random.default_rng(100 + batch)
    n, T = 2000, 70  # 2000 posts: one tile per SM of 32 posts, the last one partial
    conn = _dyadic(rng, n, 0.02)
    x = (np.round(rng.poisson(0.08, (T, batch, n)) * 0.5 * 64) / 64).astype(np.float32)
    lens = rng.integers(T // 2, T + 10, batch)
    rnn = _model(conn, n, 0, batch)
    spec = _spec(conn, n, 0)
    ost = O.init_state(spec, batch)
    for a, b in ((0, 30), (30, T)):
        sl = torch.tensor(np.clip(lens - a, 0, b - a), device="cuda")
        with torch.no_grad(), environ.context(dt=1.0):
            z, st = rnn(torch.tensor(x[a:b], device="cuda"), sample_len=sl, engine_choice=TILE, engine_stats=True)
        assert rnn.last_engine_choice == TILE
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
    assert o["spikes"].sum() > 100
    np.testing.assert_array_equal(rnn.neuron.v.cpu().numpy(), ost.v)
    np.testing.assert_array_equal(rnn.synapse.psc.cpu().numpy(), ost.psc)


@pytest.mark.parametrize("batch", [3, 64])
def test_tile_alif_with_input_layer_equals_scatter_step(batch):
    """ALIF + dense input layer: tile == two-launch scatter, bit for bit
    (dyadic weights and input), rasters, traces and final state."""
    rng = np.random.default_rng(7 + batch)
    n, T, c_in = 5000, 60, 40
    conn = _dyadic(rng, n, 0.01, exp=-6)
    w_in = (np.round(rng.normal(0, 0.3, (c_in, n)) * 64) / 64).astype(np.float32)
    x = torch.tensor(rng.poisson(0.1, (T, batch, c_in)).astype(np.float32), device="cuda")
    outs = []
    for choice in (SCATTER, TILE):
        rnn = _model(conn, n, 1, batch, c_in, w_in, names=("neuron.v", "neuron.g_k", "synapse.psc"))
        with torch.no_grad(), environ.context(dt=1.0):
            z, st = rnn(x, engine_choice=choice)
        outs.append([z.cpu().numpy(), st["neuron.v"].cpu().numpy(), st["neuron.g_k"].cpu().numpy(),
                     st["synapse.psc"].cpu().numpy(), rnn.neuron.v.cpu().numpy(), rnn.synapse.psc.cpu().numpy()])
    assert outs[0][0].sum() > 100
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def test_tile_graph_replay_equals_eager_and_bitmask_output():
    rng = np.random.default_rng(3)
    n, T, B = 3000, 300, 16
    conn = _dyadic(rng, n, 0.02)
    x = torch.tensor((np.round(rng.poisson(0.06, (T, B, n)) * 0.5 * 64) / 64).astype(np.float32), device="cuda")
    outs = []
    for graph in (False, True):
        rnn = _model(conn, n, 0, B, names=())
        rnn.cudagraph = graph
        with torch.no_grad(), environ.context(dt=1.0):
            r1, _ = rnn(x, spikes_out="bitmask", engine_choice=TILE)
            r2, _ = rnn(x, spikes_out="bitmask", engine_choice=TILE)
        outs.append((r1.cpu().numpy(), r2.cpu().numpy(), rnn.neuron.v.cpu().numpy()))
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


def test_tile_barrier_timeout_is_reported_and_the_context_stays_usable():
    """A grid-barrier wait limited to one poll gives up: the launch ends, the
    call raises, and the next call (default limit) is correct again."""
    rng = np.random.default_rng(5)
    n, T, B = 4000, 40, 4
    conn = _dyadic(rng, n, 0.02)
    x = (np.round(rng.poisson(0.08, (T, B, n)) * 0.5 * 64) / 64).astype(np.float32)
    rnn = _model(conn, n, 0, B, names=())
    rnn.engine_spin_limit = 1
    with pytest.raises(RuntimeError, match="gave up"):
        with torch.no_grad(), environ.context(dt=1.0):
            rnn(torch.tensor(x, device="cuda"), engine_choice=TILE)
    torch.cuda.synchronize()
    rnn.engine_spin_limit = 0
    init_net_state(rnn, batch_size=B, dtype=torch.float32, device="cuda")
    with torch.no_grad(), environ.context(dt=1.0):
        z, _ = rnn(torch.tensor(x, device="cuda"), engine_choice=TILE)
    spec = _spec(conn, n, 0)
    o = O.run(spec, O.init_state(spec, B), x, events=True)
    np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), o["spikes"])


def test_tile_offsets_split_rows_at_tile_boundaries():
    from btorch_b200.models.engine import tile_offsets, tile_shape

    rng = np.random.default_rng(9)
    n = 3333
    conn = SparseConn(_dyadic(rng, n, 0.01), sparse_config={"direction": "scatter"}).cuda()
    lay = conn.scatter_layout(1, 0, torch.device("cuda"))
    from btorch_b200.models._ops import pack_csr_weights

    w = pack_csr_weights(lay, conn._edge_weight().detach().float().contiguous())
    edges = torch.stack([lay.csr_dst, w.view(torch.int32)], 1).reshape(-1)
    tp, P = tile_shape(n, 8, torch.device("cuda"))
    off = tile_offsets(lay, edges, tp, P, torch.device("cuda")).cpu().numpy()
    ptr, dst = lay.csr_ptr.cpu().numpy(), lay.csr_dst.cpu().numpy()
    for r in rng.integers(0, n, 200):
        posts = dst[ptr[r]:ptr[r + 1]]
        want = ptr[r] + np.searchsorted(posts, np.arange(P + 1) * tp, side="left")
        np.testing.assert_array_equal(off[r], want)
