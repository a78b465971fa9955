"""Device compaction of bitmask rasters (bt_raster_count / bt_raster_coords)
gives exactly the host encoding of the dense spike stack."""

import numpy as np
import pytest
import torch

from btorch_b200 import _lib as L
from btorch_b200.io import from_spike_sparse, raster_to_sparse_repr, to_sparse_repr
from btorch_b200.models import environ
from tests import cases

pytestmark = pytest.mark.gpu


def bits_of(z):
    T, B, n = z.shape
    bits = torch.empty((T, B, (n + 31) // 32), dtype=torch.int32, device="cuda")
    L.check(L.lib().bt_float_to_bits(T * B, n, z.data_ptr(), bits.data_ptr(), L.stream_of(z.device)))
    return bits


def same(a, b):
    assert set(a) == set(b)
    for k in a:
        if k in ("spikes",):
            assert a[k][2] == b[k][2] and int(a[k][1]) == int(b[k][1])
        else:
            assert a[k][0] == b[k][0]
            np.testing.assert_array_equal(a[k][1], b[k][1])
            assert a[k][1].dtype == b[k][1].dtype


@pytest.mark.parametrize("shape,p", [((50, 3, 257), 0.05), ((4, 1, 32), 0.5), ((3, 2, 1000), 0.0), ((9, 70, 95), 0.2)])
def test_raster_encoding_equals_dense(shape, p):
    rng = np.random.default_rng(sum(shape))
    z = torch.tensor((rng.random(shape) < p).astype(np.float32), device="cuda")
    enc = raster_to_sparse_repr(bits_of(z), shape[2])
    same(enc, to_sparse_repr(z, ["time", "batch", "neuron"], "spikes"))
    np.testing.assert_array_equal(from_spike_sparse(enc, "spikes")[0], z.cpu().numpy())


def test_engine_bitmask_output_round_trip():
    d = cases.load("lif_dyadic_input")
    x = torch.tensor(d["x"], device="cuda")
    outs = []
    for mode in ("dense", "bitmask"):
        rnn, _ = cases.build_model(d, "cuda", "gather")
        with torch.no_grad(), environ.context(dt=1.0):
            z, _ = rnn(x, spikes_out=mode)
        outs.append(z)
    n = int(d["n"])
    same(raster_to_sparse_repr(outs[1], n), to_sparse_repr(outs[0].cpu().numpy(), ["time", "batch", "neuron"], "spikes"))
