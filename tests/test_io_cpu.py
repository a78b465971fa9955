"""Sparse spike encoding on the host: the reference's to_sparse_repr /
from_spike_sparse semantics (btorch/io/serialization.py:80-191; its tests
tests/io/test_serialization.py:45-129 check the marker attrs and round trips
through xarray, which is not installed here, so the tuples are checked
directly)."""

import numpy as np
import scipy.sparse as sp
import torch

from btorch_b200.io import from_spike_sparse, to_sparse_repr


def test_dense_raster_encoding_and_round_trip():
    rng = np.random.default_rng(0)
    z = (rng.random((7, 3, 45)) < 0.1).astype(np.float32)
    enc = to_sparse_repr(z, ["time", "batch", "neuron"], "spikes")
    idx = np.nonzero(z)
    for d, ix in zip(("time", "batch", "neuron"), idx):
        dims, vals = enc[f"spikes_idx_{d}"]
        assert dims == ["_btorch_sparse_idx_spikes"] and vals.dtype == np.int32
        np.testing.assert_array_equal(vals, ix)
    assert enc["spikes_data"][1].dtype == np.float32 and np.all(enc["spikes_data"][1] == 1.0)
    dims, nnz, attrs = enc["spikes"]
    assert dims == [] and int(nnz) == len(idx[0])
    assert attrs == {"_btorch_sparse": True, "original_shape": [7, 3, 45],
                     "original_dims": ["time", "batch", "neuron"], "original_dtype": "float32", "nnz": len(idx[0])}
    back, used = from_spike_sparse(enc, "spikes")
    np.testing.assert_array_equal(back, z)
    assert used == set(enc)


def test_scipy_and_torch_inputs():
    rng = np.random.default_rng(1)
    m = sp.random(20, 30, density=0.1, random_state=2, format="csr").astype(np.float64)
    enc = to_sparse_repr(m, ["pre", "post"], "w")
    back, _ = from_spike_sparse(enc, "w", return_sparse_2d=True)
    assert sp.issparse(back)
    np.testing.assert_allclose(back.toarray(), m.toarray())
    t = torch.tensor((rng.random((4, 9)) < 0.3).astype(np.int64))
    enc = to_sparse_repr(t, ["time", "neuron"], "s")
    assert enc["s"][2]["original_dtype"] == "int64"
    np.testing.assert_array_equal(from_spike_sparse(enc, "s")[0], t.numpy())


def test_empty():
    enc = to_sparse_repr(np.zeros((2, 2, 5), np.float32), ["time", "batch", "neuron"], "z")
    assert int(enc["z"][1]) == 0 and enc["z_idx_time"][1].size == 0
    np.testing.assert_array_equal(from_spike_sparse(enc, "z")[0], np.zeros((2, 2, 5), np.float32))


def test_constraint_groups_follow_reference_order():
    """SparseConstrainedConn maps every stored nonzero (canonical order) to the
    reference's 0-based group (fixture from the reference)."""
    import scipy.sparse as sp

    from btorch_b200.models import SparseConstrainedConn
    from tests import cases

    d = cases.load("constrained_spmm")
    C = sp.coo_array((d["C_data"], (d["C_row"], d["C_col"])), shape=d["W"].shape)
    m = SparseConstrainedConn(sp.coo_array(d["W"]), C)
    np.testing.assert_array_equal(m._constraint_scatter_indices.numpy(), d["group"])
    assert m.magnitude.shape == (3,) and torch.all(m.magnitude == 1)
