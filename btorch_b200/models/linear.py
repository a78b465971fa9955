"""Connectivity layers (API of btorch/models/linear.py).

SparseConn keeps the reference's buffers and state_dict keys: ``indices``
(2, nnz) int64 in canonical (post, src) order, ``magnitude`` (Parameter, same
order), optional ``bias`` and the Dale sign ``initial_sign``
(linear.py:252-319, 535-591).  Its forward runs the event-driven sm_100a
sparse product (ordered gather or scatter, see _sparse_config); the device
layout (CSC/CSR views) is rebuilt from ``indices`` at construction and on
load_state_dict (linear.py:351-373).
"""

from __future__ import annotations

from typing import Any

import numpy as np
import scipy.sparse
import torch
import torch.nn as nn

from .. import config as bt_config
from .._sparse_config import BACKEND_NAMES, SparseBackendConfig
from . import _ops
from .constrain import HasConstraint
from ._ops import SparseLayout, build_layout, pack_csr_weights


def _resolve_sparse_backend(backend: str | None) -> str:
    if backend is None:
        return bt_config.sparse.selected or "b200"
    b = backend.lower()
    if b not in BACKEND_NAMES:
        raise ValueError(f"sparse_backend must be one of {BACKEND_NAMES}, got '{backend}'.")
    return b


def available_sparse_backends(*, include_experimental: bool = False) -> list[str]:
    """Every name selects the same sm_100a implementation."""
    return list(BACKEND_NAMES)


class DenseConn(nn.Linear, HasConstraint):
    """Dense connection y = x @ W (+ b) with optional mask and Dale sign
    (linear.py:163-228).  Inside the fused engine its projection runs as an
    event-driven kernel over the nonzero inputs; stepped alone it is nn.Linear."""

    def __init__(self, in_features: int, out_features: int, weight=None, bias=None, mask=None,
                 enforce_dale: bool = False, device=None, dtype=None):
        super().__init__(in_features, out_features, bias=bias is not None, device=device, dtype=dtype)
        if weight is not None:
            self.weight.data = torch.as_tensor(weight).T.to(self.weight.dtype).contiguous()
        if bias is not None:
            self.bias.data = torch.as_tensor(bias).to(self.weight.dtype)
        if mask is not None:
            if isinstance(mask, (int, float)):
                mask = (torch.rand(self.weight.shape, device=device, dtype=dtype) < mask).to(self.weight.dtype)
            self.register_buffer("mask", mask)
        else:
            self.mask = None
        if enforce_dale:
            self.register_buffer("initial_sign", torch.sign(self.weight.data))
        else:
            self.initial_sign = None

    def constrain(self, *args, **kwargs):
        if self.mask is not None:
            self.weight.data *= self.mask
        if self.initial_sign is not None:
            self.weight.data = (self.weight.data * self.initial_sign).relu() * self.initial_sign


class BaseSparseConn(nn.Module):
    """x @ conn for a fixed sparse conn of shape (in_features, out_features)."""

    def __init__(self, conn, bias=None, sparse_backend: str | None = None,
                 sparse_config: SparseBackendConfig | dict[str, Any] | None = None, device=None, dtype=None):
        super().__init__()
        self.sparse_backend = _resolve_sparse_backend(sparse_backend)
        self.sparse_config = bt_config.sparse.resolve(self.sparse_backend, sparse_config)
        self._prepared_sparse_weight: torch.Tensor | None = None
        self._sparse_prepare_depth = 0
        if not isinstance(conn, scipy.sparse.coo_array):
            conn = scipy.sparse.coo_array(conn) if isinstance(conn, np.ndarray) else conn.tocoo()
        self.in_features, self.out_features = (int(s) for s in conn.shape)
        self.shape = (self.in_features, self.out_features)
        c = conn.T
        c.sum_duplicates()
        indices = torch.stack([torch.tensor(c.row, dtype=torch.long, device=device),
                               torch.tensor(c.col, dtype=torch.long, device=device)])
        self.register_buffer("indices", indices)
        value = torch.tensor(c.data, dtype=dtype or torch.float32, device=device)
        self.bias = nn.Parameter(bias) if bias is not None else None
        self._layout: SparseLayout | None = None
        self._engine_layouts: dict = {}
        self._init_weights(value)

    # -- layout ------------------------------------------------------------
    def layout(self, device=None) -> SparseLayout:
        """CSC/CSR device views of `indices` (built once per device)."""
        dev = torch.device(device) if device is not None else self.indices.device
        if self._layout is None or self._layout.csc_ptr.device != dev:
            lay = build_layout(self.indices, self.in_features, self.out_features, 1)
            self._layout = lay.to(dev)
        return self._layout

    def engine_layout(self, n_bins: int, uniform_delay: int, device) -> SparseLayout:
        """Layout with delay bins decoded: rows are pre * n_bins + bin of a
        delay-expanded conn, or every edge carries `uniform_delay` (DelayedPSC)."""
        dev = torch.device(device)
        key = (n_bins, uniform_delay, str(dev))
        lay = self._engine_layouts.get(key)
        if lay is None:
            if uniform_delay:
                R = uniform_delay + 1
                idx = torch.stack([self.indices[0], self.indices[1] * R + uniform_delay])
                lay = build_layout(idx, self.in_features, self.out_features, R)
            else:
                lay = build_layout(self.indices, self.in_features // n_bins, self.out_features, n_bins)
            lay = lay.to(dev)
            self._engine_layouts[key] = lay
        return lay

    def scatter_layout(self, n_bins: int, uniform_delay: int, device) -> SparseLayout:
        """CSR over the rows pre * n_bins + bin of the delay-expanded matrix
        (the fused engine's scatter mode), with the delay bins that hold edges
        (`bin_lo`, `bin_hi`) and the mean length of a non-empty row."""
        dev = torch.device(device)
        key = ("scatter", n_bins, uniform_delay, str(dev))
        lay = self._engine_layouts.get(key)
        if lay is None:
            if uniform_delay:
                R = uniform_delay + 1
                idx = torch.stack([self.indices[0], self.indices[1] * R + uniform_delay])
                lay = build_layout(idx, self.in_features * R, self.out_features, 1)
            else:
                lay = build_layout(self.indices, self.in_features, self.out_features, 1)
            rows = (lay.csr_ptr[1:] - lay.csr_ptr[:-1]).view(-1, n_bins)
            per_bin = np.nonzero(rows.sum(0).numpy())[0]
            bins = (int(per_bin[0]), int(per_bin[-1])) if per_bin.size else (0, 0)
            mean_row = lay.nnz / max(1, int((rows > 0).sum()))
            lay = lay.to(dev)
            lay.bin_lo, lay.bin_hi = bins
            lay.mean_row = mean_row
            self._engine_layouts[key] = lay
        return lay

    def _apply(self, fn, recurse=True):
        self._prepared_sparse_weight = None
        self._sparse_prepare_depth = 0
        out = super()._apply(fn, recurse=recurse)
        self._layout = None
        self._engine_layouts = {}
        return out

    def _load_from_state_dict(self, state_dict, prefix, local_metadata, strict, missing_keys, unexpected_keys,
                              error_msgs):
        super()._load_from_state_dict(state_dict, prefix, local_metadata, strict, missing_keys, unexpected_keys,
                                      error_msgs)
        self._prepared_sparse_weight = None
        self._sparse_prepare_depth = 0
        self._layout = None
        self._engine_layouts = {}

    def _edge_weight(self) -> torch.Tensor:
        """The effective weight, one value per stored nonzero in canonical
        order.  The kernels index it by edge, so a weight whose length is not
        the number of stored nonzeros (a mismatched checkpoint, a reassigned
        magnitude) is refused here, where the reference's
        torch.sparse_coo_tensor raises."""
        w = self._get_effective_weight()
        if w.numel() != self.indices.shape[1]:
            raise RuntimeError(f"{type(self).__name__} has {self.indices.shape[1]} stored nonzeros but "
                               f"{w.numel()} weights.")
        return w

    # -- prepare scope (linear.py:375-415) -----------------------------------
    def prepare_sparse(self, batch_size: int | None = None) -> None:
        """Pack the effective weight into CSR order once for a multi-step run."""
        if self._prepared_sparse_weight is None and self.indices.is_cuda:
            w = self._edge_weight()
            self._prepared_sparse_weight = pack_csr_weights(self.layout(w.device), w.float())
        self._sparse_prepare_depth += 1

    def finish_sparse(self) -> None:
        if self._sparse_prepare_depth <= 0:
            raise RuntimeError("finish_sparse called without prepare_sparse.")
        self._sparse_prepare_depth -= 1
        if self._sparse_prepare_depth == 0:
            self._prepared_sparse_weight = None

    def _init_weights(self, value):
        raise NotImplementedError

    def _get_effective_weight(self):
        raise NotImplementedError

    def get_sparse_matrix(self) -> torch.Tensor:
        v = self._get_effective_weight()
        idx = torch.stack([self.indices[1], self.indices[0]])
        return torch.sparse_coo_tensor(idx, v, size=(self.in_features, self.out_features), is_coalesced=True)

    def direction(self, batch: int) -> str:
        cfg = self.sparse_config
        if cfg.deterministic:
            return "gather"
        if cfg.direction != "auto":
            return cfg.direction
        return "gather" if self.indices.shape[1] * max(1, batch) <= cfg.gather_max_nnz_per_step else "scatter"

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        no_batch = x.ndim == 1
        if no_batch:
            x = x[None, :]
        if x.shape[-1] != self.in_features:
            # (the reference's torch.sparse.mm raises here; the kernels would
            # index x and the source rows by the layout's width)
            raise RuntimeError(f"SparseConn takes {self.in_features} input features, got shape {tuple(x.shape)}.")
        leading = x.shape[:-1]
        x2 = x.reshape(-1, x.shape[-1])
        w = self._edge_weight()
        if w.dtype != torch.float32:
            raise TypeError("SparseConn supports float32 only.")
        lay = self.layout(x2.device) if x2.is_cuda else None
        if lay is None:
            raise RuntimeError("SparseConn requires CUDA tensors (there is no CPU path).")
        w_csr = self._prepared_sparse_weight if not w.requires_grad or not torch.is_grad_enabled() else None
        out = _ops.sparse_mm(x2, w, lay, self.direction(x2.shape[0]), w_csr)
        out = out.reshape(*leading, self.out_features)
        if no_batch:
            out = out[0]
        if self.bias is not None:
            out = out + self.bias
        return out


class SparseConn(BaseSparseConn, HasConstraint):
    """Sparse linear map with a learnable magnitude per stored nonzero and an
    optional Dale sign (linear.py:535-591)."""

    @classmethod
    def from_canonical(cls, post: np.ndarray, src: np.ndarray, values: np.ndarray, shape: tuple[int, int],
                       **kwargs) -> "SparseConn":
        """Build from arrays already in canonical (post, src) order -- the
        order ``indices`` stores -- without a scipy round trip (large
        connectomes).  shape = (in_features, out_features)."""
        post = np.asarray(post)
        src = np.asarray(src)
        key_ok = np.all((post[1:] > post[:-1]) | ((post[1:] == post[:-1]) & (src[1:] > src[:-1])))
        if post.size and not key_ok:
            raise ValueError("from_canonical needs strictly increasing (post, src) pairs")
        stub = scipy.sparse.coo_array((np.zeros(0, np.float32), (np.zeros(0, np.int64), np.zeros(0, np.int64))),
                                      shape=shape)
        m = cls(stub, **kwargs)
        dev = m.indices.device
        m.indices = torch.stack([torch.as_tensor(post, dtype=torch.long), torch.as_tensor(src, dtype=torch.long)]).to(dev)
        value = torch.as_tensor(np.asarray(values), dtype=m.magnitude.dtype).to(dev)
        if getattr(m, "enforce_dale", False):
            m.initial_sign = torch.sign(value)
        m.magnitude = nn.Parameter(value)
        m._layout = None
        m._engine_layouts = {}
        return m

    def __init__(self, conn, bias=None, enforce_dale: bool = True, sparse_backend: str | None = None,
                 sparse_config=None, device=None, dtype=None):
        self.enforce_dale = enforce_dale
        super().__init__(conn, bias=bias, sparse_backend=sparse_backend, sparse_config=sparse_config,
                         device=device, dtype=dtype)

    def _init_weights(self, value):
        if self.enforce_dale:
            self.register_buffer("initial_sign", torch.sign(value), persistent=False)
        self.magnitude = nn.Parameter(value)

    def _get_effective_weight(self):
        return self.magnitude

    def constrain(self, *args, **kwargs):
        if self.enforce_dale:
            self.magnitude.data = (self.magnitude * self.initial_sign).relu() * self.initial_sign


class SparseConstrainedConn(BaseSparseConn, HasConstraint):
    """Sparse linear layer whose weights share learnable magnitudes by
    constraint group (btorch/models/linear.py:594-867): effective weight of
    stored nonzero e = initial_weight[e] * magnitude[group[e]], groups given by
    a constraint matrix of 1-based group ids with the sparsity of `conn`.
    Runs on the same kernels as SparseConn (the effective weight is formed on
    the device once per call or run); the gradient of a magnitude is the sum
    over its group of initial_weight times the per-nonzero weight gradient."""

    def __init__(self, conn, constraint, enforce_dale: bool = True, bias=None, sparse_backend: str | None = None,
                 sparse_config=None, device=None, dtype=None, persist_initial_weight: bool = False):
        self.enforce_dale = enforce_dale
        self.persist_initial_weight = persist_initial_weight
        self.constraint_info = None
        c = constraint.T
        if not isinstance(c, scipy.sparse.coo_array):
            c = scipy.sparse.coo_array(c)
        c.eliminate_zeros()
        if c.nnz and (c.data.min() < 1 or not np.all(np.mod(c.data, 1) == 0)):
            # ids index the magnitudes on the device (id - 1)
            raise ValueError("constraint group ids must be integers >= 1 (0 means no constraint)")
        self._constraint_matrix = c
        super().__init__(conn, bias=bias, sparse_backend=sparse_backend, sparse_config=sparse_config,
                         device=device, dtype=dtype)

    def _init_weights(self, value):
        self.register_buffer("initial_weight", value, persistent=self.persist_initial_weight)
        n_groups = int(self._constraint_matrix.data.max()) if self._constraint_matrix.nnz else 0
        self.magnitude = nn.Parameter(torch.ones(n_groups, dtype=value.dtype, device=value.device))
        self.register_buffer("_constraint_scatter_indices",
                             torch.as_tensor(self._group_of_nonzeros(), dtype=torch.long, device=value.device),
                             persistent=False)

    def _group_of_nonzeros(self) -> np.ndarray:
        """0-based group id of every stored nonzero (canonical order), looked
        up in the constraint matrix by (post, src) key."""
        idx = self.indices.cpu().numpy()
        n_src = max(self.in_features, 1)
        key = idx[0].astype(np.int64) * n_src + idx[1]
        c = self._constraint_matrix
        ckey = c.row.astype(np.int64) * n_src + c.col
        order = np.argsort(ckey, kind="stable")
        ckey, gid = ckey[order], c.data[order].astype(np.int64)
        pos = np.searchsorted(ckey, key)
        ok = (pos < ckey.size) & (ckey[np.minimum(pos, max(ckey.size - 1, 0))] == key) if ckey.size else \
            np.zeros(key.size, bool)
        if not ok.all():
            raise AssertionError("Constraint missing for some connections.")
        return gid[pos] - 1

    def reset_parameters(self) -> None:
        nn.init.ones_(self.magnitude)

    def _get_effective_weight(self):
        return self.initial_weight * self.magnitude[self._constraint_scatter_indices]

    def constrain(self, *args, **kwargs):
        if self.enforce_dale:
            self.magnitude.data = self.magnitude.relu()

    @classmethod
    def from_hetersynapse(cls, conn, constraint, receptor_type_index, enforce_dale: bool = True, bias=None,
                          sparse_backend=None, sparse_config=None, device=None, dtype=None,
                          persist_initial_weight: bool = False) -> "SparseConstrainedConn":
        inst = cls(conn=conn, constraint=constraint, enforce_dale=enforce_dale, bias=bias,
                   sparse_backend=sparse_backend, sparse_config=sparse_config, device=device, dtype=dtype,
                   persist_initial_weight=persist_initial_weight)
        inst.constraint_info = {"receptor_type_index": receptor_type_index}
        return inst

    def get_group_info(self, include_weights: bool = False):
        import pandas as pd

        gid = self._constraint_scatter_indices
        n_groups = len(self.magnitude)
        counts = torch.bincount(gid, minlength=n_groups).cpu().tolist()
        mags = self.magnitude.detach().cpu().tolist()
        rows = []
        for g in range(n_groups):
            info = {"group_id": g, "num_connections": counts[g], "current_magnitude": mags[g]}
            if include_weights:
                w = self.initial_weight[gid == g]
                info["mean_initial_weight"] = w.mean().item()
                info["std_initial_weight"] = w.std(unbiased=False).item()
            rows.append(info)
        df = pd.DataFrame(rows)
        if self.constraint_info is not None:
            ri = self.constraint_info["receptor_type_index"]
            if len(ri) == n_groups:
                df = pd.concat([df, ri.reset_index(drop=True)], axis=1)
        return df

    def set_group_magnitude(self, group_id: int | None = None, receptor_pair=None, value=1.0):
        if (group_id is None) == (receptor_pair is None):
            raise ValueError("Exactly one of group_id or receptor_pair must be specified")
        if receptor_pair is not None:
            if self.constraint_info is None:
                raise ValueError("receptor_pair can only be used if created via from_hetersynapse")
            ri = self.constraint_info["receptor_type_index"]
            if "pre_receptor_type" not in ri.columns:
                raise ValueError("receptor_pair requires neuron mode (pre_receptor_type, post_receptor_type)")
            group_id = ri.set_index(["pre_receptor_type", "post_receptor_type"]).loc[tuple(receptor_pair),
                                                                                    "receptor_index"]
        if isinstance(value, (int, float)):
            value = torch.tensor(value, dtype=self.magnitude.dtype, device=self.magnitude.device)
        self.magnitude.data[group_id] = value

    def get_weights_by_group(self) -> dict:
        gid = self._constraint_scatter_indices
        return {g: self.initial_weight[gid == g] * self.magnitude[g] for g in range(len(self.magnitude))}


__all__ = ["DenseConn", "BaseSparseConn", "SparseConn", "SparseConstrainedConn", "available_sparse_backends"]
