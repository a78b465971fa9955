"""Spike-raster serialisation (API of btorch/io/serialization.py:80-200).

`to_sparse_repr` / `from_spike_sparse` keep the reference's sparse COO
encoding -- one int32 index array per dimension in row-major order, a data
array of the original dtype and a scalar marker carrying shape, dims, dtype
and nnz -- as plain (dims, values[, attrs]) tuples, the form the reference
hands to xarray.Dataset.  `raster_to_sparse_repr` produces the same encoding
directly from the engine's bitmask raster (RecurrentNN(..., spikes_out=
"bitmask")), compacted on the device by bt_raster_count / bt_raster_coords,
so a (T, B, N) fp32 stack is never materialised.
"""

from __future__ import annotations

from collections.abc import Mapping, Sequence
from typing import Any

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib as L


def _marker(nnz: int, shape, dims, dtype) -> tuple:
    return ([], np.int32(nnz), {"_btorch_sparse": True, "original_shape": list(shape),
                                "original_dims": list(dims), "original_dtype": str(np.dtype(dtype)),
                                "nnz": int(nnz)})


def _encode(indices, data, shape, var_dims, var_name, dtype) -> dict[str, Any]:
    sparse_dim = f"_btorch_sparse_idx_{var_name}"
    out = {f"{var_name}_idx_{d}": ([sparse_dim], np.asarray(ix).astype(np.int32)) for d, ix in zip(var_dims, indices)}
    out[f"{var_name}_data"] = ([sparse_dim], np.asarray(data))
    out[var_name] = _marker(len(data), shape, var_dims, dtype)
    return out


def to_sparse_repr(val, var_dims: Sequence[str], var_name: str) -> dict[str, Any]:
    """Sparse COO encoding of a dense (numpy / torch) or scipy sparse array,
    as the reference computes it (serialization.py:80-141)."""
    if torch.is_tensor(val):
        val = val.detach().cpu().numpy()
    if sp.issparse(val):
        coo = val.tocoo()
        return _encode((coo.row, coo.col), coo.data, val.shape, var_dims, var_name, val.dtype)
    val = np.asarray(val)
    idx = np.nonzero(val)
    return _encode(idx, val[idx], val.shape, var_dims, var_name, val.dtype)


def raster_to_sparse_repr(raster: torch.Tensor, n: int, var_name: str = "spikes",
                          var_dims: Sequence[str] = ("time", "batch", "neuron"),
                          dtype=np.float32) -> dict[str, Any]:
    """The encoding of the spike stack a bitmask raster [T, B, ceil(n/32)]
    int32 stands for (values 1 of `dtype`), computed on the raster's device."""
    if not (torch.is_tensor(raster) and raster.is_cuda and raster.dtype == torch.int32 and raster.ndim == 3):
        raise TypeError("raster must be a CUDA int32 tensor [T, B, ceil(n/32)]")
    T, B, W = raster.shape
    if W != (n + 31) // 32:
        raise ValueError(f"raster has {W} words per row, n={n} needs {(n + 31) // 32}")
    bits = raster.contiguous()
    dev = bits.device
    s = L.stream_of(dev)
    rows = T * B
    counts = torch.empty(max(rows, 1), dtype=torch.int64, device=dev)
    L.check(L.lib().bt_raster_count(rows, n, bits.data_ptr(), counts.data_ptr(), s), "bt_raster_count")
    offsets = torch.zeros(rows + 1, dtype=torch.int64, device=dev)
    if rows:
        torch.cumsum(counts[:rows], 0, out=offsets[1:])
    nnz = int(offsets[-1])
    idx = torch.empty((3, max(nnz, 1)), dtype=torch.int32, device=dev)
    L.check(L.lib().bt_raster_coords(rows, B, n, bits.data_ptr(), offsets.data_ptr(), idx[0].data_ptr(),
                                     idx[1].data_ptr(), idx[2].data_ptr(), s), "bt_raster_coords")
    ix = idx[:, :nnz].cpu().numpy()
    return _encode((ix[0], ix[1], ix[2]), np.ones(nnz, dtype=dtype), (T, B, n), var_dims, var_name, dtype)


def _values(entry):
    if hasattr(entry, "values") and not isinstance(entry, tuple):
        return np.asarray(entry.values), dict(getattr(entry, "attrs", {}))
    return np.asarray(entry[1]), (dict(entry[2]) if len(entry) > 2 else {})


def from_spike_sparse(ds: Mapping, var_name: str, return_sparse_2d: bool = False):
    """Dense (or 2-D scipy COO) array from the encoding, and the names used
    (serialization.py:144-191).  `ds` maps names to (dims, values[, attrs])
    tuples or to xarray-like variables with .values and .attrs."""
    _, attrs = _values(ds[var_name])
    shape = tuple(attrs["original_shape"])
    dims = attrs["original_dims"]
    dtype = np.dtype(attrs["original_dtype"])
    used = {var_name}
    indices = []
    for d in dims:
        name = f"{var_name}_idx_{d}"
        indices.append(_values(ds[name])[0])
        used.add(name)
    data = _values(ds[f"{var_name}_data"])[0]
    used.add(f"{var_name}_data")
    if return_sparse_2d and len(shape) == 2:
        return sp.coo_array((data, (indices[0], indices[1])), shape=shape), used
    out = np.zeros(shape, dtype=dtype)
    out[tuple(indices)] = data
    return out, used
