"""Parity at the benchmark configurations' own sizes: the engine on each
workload's full network and seeded input (the generators bench.py times)
against the CPU oracle (event-driven push, bit-identical to the reference's
per-synapse chain; pinned in tests/test_oracle_golden.py).

  plain       LIF N 4096, p 0.02, lognormal E/I weights, 1000 Poisson
              channels through a dense input layer, batch 1, T 1000: the
              ordered gather and the single-cluster engine bit for bit over
              all 1000 steps; the scatter
              (arrival-order sums of non-dyadic weights) within rel 1e-5
              until the first spike divergence.
  connectome  LIF N 140000, 48.8M synapses (dyadic counts x 2^-6), delays
              1..20, batch 8: the scatter bit for bit over the first 200
              steps (rasters and final state) -- exact partial sums.
  batched     ALIF N 65536, in-degree 500, batch 64, 2000 input channels:
              the first 100 steps (the start-up burst, dense steps
              included) within rel 1e-5 per sample until that sample's
              first spike divergence.
And the plain single-request step (batch 1, eager) of the connectome
workload produces sample 0's raster of the batched run.
"""

import numpy as np
import pytest
import torch

import bench

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def _workload(name, steps):
    cfg = dict(bench.CONFIGS[name], t_max=steps)
    net = bench.make_network(cfg, 0)
    x, lens = bench.make_inputs(cfg, 0, DEV)
    return cfg, net, x, lens


@pytest.mark.parametrize("mode", ["gather", "cluster"])
def test_plain_ordered_modes_bitwise_all_steps(mode):
    """The warp-per-post gather and the single-cluster engine (the tuner's
    choice for this workload), each over all 1000 steps."""
    cfg, net, x, lens = _workload("plain", 1000)
    r = bench.parity_bitwise("plain", cfg, net, x, lens, DEV, 1000, "gather", choice=mode)
    assert r["direction"] == f"gather ({mode})", r
    assert r["spikes"] > 0
    assert r["check"] == "bitwise", r


def test_plain_scatter_within_tolerance_until_divergence():
    cfg, net, x, lens = _workload("plain", 1000)
    r = bench.parity_tolerance("plain", cfg, net, x, lens, DEV, 1000, "scatter")
    assert r["check"].startswith("within"), r
    assert r["first_divergence"] >= 2, r


def test_connectome_scatter_bitwise_first_200_steps():
    cfg, net, x, lens = _workload("connectome", 200)
    r = bench.parity_bitwise("connectome", cfg, net, x, lens, DEV, 200, "scatter")
    assert r["direction"].startswith("scatter")
    assert r["spikes"] > 1000
    assert r["check"] == "bitwise", r


def test_batched_alif_first_100_steps_within_tolerance():
    cfg, net, x, lens = _workload("batched", 100)
    r = bench.parity_tolerance("batched", cfg, net, x, lens, DEV, 100, "scatter")
    assert r["check"].startswith("within"), r
    assert r["spikes"] > 10_000_000  # the burst: dense steps run


def test_plain_step_raster_is_sample_zero_of_the_batch():
    cfg, net, x, lens = _workload("connectome", 300)
    z, _, _, _ = bench.engine_window(cfg, net, x, lens, DEV, "scatter", 300)
    one = dict(cfg, batch=1)
    z1, _, _, _ = bench.engine_window(one, net, x[:, :1].contiguous(), lens[:1], DEV, "scatter", 300,
                                      cudagraph=False)
    assert z[:, 0].sum() > 0
    np.testing.assert_array_equal(z1[:, 0], z[:, 0])
