"""CUDA-graph replay (RecurrentNN(cudagraph=True)) gives the eager results bit
for bit: the fused engine's captured chunks across full chunks, a ragged last
chunk and consecutive calls, and the per-module path through CudaGraphRunner."""

import numpy as np
import pytest
import torch

from btorch_b200.models import engine, environ
from tests import cases

pytestmark = pytest.mark.gpu
DEV = "cuda"
MODES = ["gather", "pull", "scatter"]


def _run(d, direction, graph, splits, chunk=None, fused=True, sample_len=None):
    rnn, psc_name = cases.build_model(d, DEV, direction)
    rnn.cudagraph = graph
    rnn.fused = fused
    x = torch.tensor(d["x"], device=DEV)
    zs, vs, stats = [], [], []
    with torch.no_grad(), environ.context(dt=float(d["dt"])):
        for a, b in zip([0] + splits, splits + [len(x)]):
            kw = {} if not fused else {"engine_chunk": chunk, "engine_stats": True, "sample_len": sample_len}
            z, st = rnn(x[a:b], **kw)
            zs.append(z.cpu().numpy())
            vs.append(st["neuron.v"].cpu().numpy())
            if fused:
                stats.append(rnn.last_engine_stats.cpu().numpy())
    return rnn, np.concatenate(zs), np.concatenate(vs), stats, rnn.neuron.v.cpu().numpy()


@pytest.mark.parametrize("direction", MODES)
@pytest.mark.parametrize("name", ["lif_dyadic_input", "delayed_psc", "hetero_delay", "alif_exppsc"])
def test_fused_graph_equals_eager(name, direction):
    d = cases.load(name)
    _, z0, v0, s0, vf0 = _run(d, direction, False, [50])
    rnn, z1, v1, s1, vf1 = _run(d, direction, True, [50], chunk=16)
    if direction == "scatter" and name == "alif_exppsc":
        # non-dyadic weights: the scatter's float atomics sum in arrival order,
        # so two eager runs already differ in the last bits
        np.testing.assert_allclose(v1[:20], v0[:20], rtol=1e-5, atol=1e-5)
    else:
        np.testing.assert_array_equal(z1, z0)
        np.testing.assert_array_equal(v1, v0)
        np.testing.assert_array_equal(vf1, vf0)
        for a, b in zip(s0, s1):
            np.testing.assert_array_equal(a, b)
    entries = list(engine.graph_entries(rnn).values())
    assert len(entries) == 1
    # both calls start with a full chunk: one capture, the rest replays
    assert entries[0].captures == 1 and entries[0].replays >= 2


@pytest.mark.parametrize("direction", MODES)
def test_fused_graph_uneven_lengths(direction):
    d = cases.load("lif_dyadic_soft")
    lens = torch.tensor([120, 47, 1, 90])
    _, z0, v0, _, vf0 = _run(d, direction, False, [], sample_len=lens)
    _, z1, v1, _, vf1 = _run(d, direction, True, [], chunk=16, sample_len=lens)
    np.testing.assert_array_equal(z1, z0)
    np.testing.assert_array_equal(vf1, vf0)


def test_fused_graph_recaptures_on_new_state_shape():
    d = cases.load("lif_dyadic_soft")
    rnn, _ = cases.build_model(d, DEV, "gather")
    rnn.cudagraph = True
    x = torch.tensor(d["x"], device=DEV)
    from btorch_b200.models.functional import init_net_state

    with torch.no_grad(), environ.context(dt=1.0):
        rnn(x, engine_chunk=16)
        init_net_state(rnn, batch_size=2, dtype=torch.float32, device=DEV)
        z, _ = rnn(x[:, :2], engine_chunk=16)
    assert len(engine.graph_entries(rnn)) == 2
    ref_z = cases.spikes(d)
    np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), ref_z[:, :2])


def test_modular_graph_equals_eager():
    d = cases.load("delayed_psc")
    _, z0, v0, _, vf0 = _run(d, "gather", False, [60], fused=False)
    rnn, z1, v1, _, vf1 = _run(d, "gather", True, [60], fused=False)
    assert rnn.last_path == "modular"
    np.testing.assert_array_equal(z1, z0)
    np.testing.assert_array_equal(v1, v0)
    np.testing.assert_array_equal(vf1, vf0)
    assert len(rnn._cudagraph_runner.entries) == 1


def test_graph_refuses_gradients():
    d = cases.load("lif_dyadic_soft")
    rnn, _ = cases.build_model(d, DEV, "gather")
    rnn.cudagraph = True
    rnn.neuron.v.requires_grad_(False)
    x = torch.tensor(d["x"], device=DEV, requires_grad=True)
    with pytest.raises(RuntimeError, match="inference-only"):
        rnn(x)


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("name", ["lif_dyadic_input", "hetero_delay"])
def test_host_input_streams_equal_device_input(name, graph):
    """Host-resident input (pinned or not): chunks stream to the device on a
    copy stream and the outputs stream back; results equal the device-input
    run bit for bit, outputs on the host."""
    d = cases.load(name)
    outs = {}
    for where in ("cuda", "cpu", "pinned"):
        rnn, _ = cases.build_model(d, DEV, "scatter")
        rnn.cudagraph = graph
        x = torch.tensor(d["x"])
        x = x.to(DEV) if where == "cuda" else (x.pin_memory() if where == "pinned" else x)
        with torch.no_grad(), environ.context(dt=float(d["dt"])):
            z, st = rnn(x, engine_chunk=24, engine_stats=True)
            stats = rnn.last_engine_stats.cpu().numpy()
            r, _ = rnn(x[:50], spikes_out="bitmask", engine_chunk=24)
        assert z.device.type == ("cuda" if where == "cuda" else "cpu")
        assert r.device.type == z.device.type
        outs[where] = (z.cpu().numpy(), st["neuron.v"].cpu().numpy(), stats, r.cpu().numpy(),
                       rnn.neuron.v.cpu().numpy())
    for where in ("cpu", "pinned"):
        for a, b in zip(outs["cuda"], outs[where]):
            np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(outs["cuda"][0].astype(np.uint8), cases.spikes(d))
