"""The continuous-batching server on the GPU: requests of different networks,
lengths and arrival times share launches, and every request's spike raster
equals the same request run alone through the module API (batch 1)."""

import numpy as np
import pytest
import torch

from btorch_b200.models import environ
from btorch_b200.serving import NetworkPool, SimRequest, SimulationServer
from tests import cases

pytestmark = pytest.mark.gpu
DEV = "cuda"


def alone(d, direction, stim):
    """Raster of one request run by itself: a fresh batch-1 model, eager."""
    rnn, _ = cases.build_model(dict(d, batch=np.int64(1)), DEV, direction)
    rnn.update_state_names = ()
    with torch.no_grad(), environ.context(dt=float(d["dt"])):
        raster, _ = rnn(stim[:, None].to(DEV), spikes_out="bitmask")
    return raster[:, 0].cpu().numpy()


@pytest.mark.parametrize("direction", ["gather", "pull", "scatter"])
def test_served_results_equal_alone(direction):
    specs = {"het": cases.load("hetero_delay"), "inp": cases.load("lif_dyadic_input")}
    pools = {}
    for name, d in specs.items():
        rnn, _ = cases.build_model(dict(d, batch=np.int64(3)), DEV, direction)
        rnn.update_state_names = ()
        pools[name] = NetworkPool(name, rnn, slots=3, chunk=16, device=DEV, cudagraph=True)
    rng = np.random.default_rng(7)
    reqs = []
    for i in range(14):
        name = "het" if i % 2 else "inp"
        d = specs[name]
        T = int(rng.integers(5, 110))
        b = int(rng.integers(0, d["x"].shape[1]))
        t0 = int(rng.integers(0, d["x"].shape[0] - T + 1))
        stim = torch.tensor(d["x"][t0:t0 + T, b])
        reqs.append(SimRequest(network=name, stimulus=stim, arrival=0.0005 * i, rid=i))
    budget = sum(pools[r.network].request_bytes(r) for r in reqs) // 2
    server = SimulationServer(pools, hbm_budget_bytes=budget)
    stims = {r.rid: r.stimulus.clone() for r in reqs}
    rep = server.run(reqs)
    assert sorted(r.rid for r in rep.requests) == list(range(14))
    assert all(p.ticks > 0 for p in pools.values())
    for r in rep.requests:
        want = alone(specs[r.network], direction, stims[r.rid])
        np.testing.assert_array_equal(r.raster.cpu().numpy(), want, err_msg=f"request {r.rid}")
    s = rep.summary()
    assert s["p50_ms"] <= s["p99_ms"] and s["events_per_s"] > 0


@pytest.mark.parametrize("limit", ["budget", "slots"])
def test_admission_holds_a_request_until_budget_or_slot_frees(limit):
    """Two requests arrive together.  Either the HBM budget fits only one of
    them (two slots free) or the network has one slot: the second waits in
    the queue until the first has retired, then runs, and each raster equals
    the request run alone."""
    d = cases.load("lif_dyadic_input")
    slots = 2 if limit == "budget" else 1
    rnn, _ = cases.build_model(dict(d, batch=np.int64(slots)), DEV, "scatter")
    rnn.update_state_names = ()
    pool = NetworkPool("inp", rnn, slots=slots, chunk=16, device=DEV, cudagraph=True)
    stims = [torch.tensor(d["x"][:100, 0]), torch.tensor(d["x"][10:90, 1])]
    reqs = [SimRequest(network="inp", stimulus=s.clone(), arrival=0.0, rid=i) for i, s in enumerate(stims)]
    need = max(pool.request_bytes(r) for r in reqs)
    budget = need if limit == "budget" else 10 * need
    rep = SimulationServer({"inp": pool}, hbm_budget_bytes=budget).run(reqs)
    done = {r.rid: r for r in rep.requests}
    assert sorted(done) == [0, 1]
    first, second = sorted(done.values(), key=lambda r: r.t_admit)
    assert second.t_admit >= first.t_done  # held back until the first one retired
    for r in rep.requests:
        np.testing.assert_array_equal(r.raster.cpu().numpy(), alone(d, "scatter", stims[r.rid]),
                                      err_msg=f"request {r.rid}")
