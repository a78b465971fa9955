"""Connectome input format feeding the recurrent step.

API of btorch/connectome/connection.py:

* make_sparse_mat (:15-39): connection table -> (pre, post) COO, duplicate
  pairs summed, entries in (pre, post) order.
* make_hetersynapse_conn (:218-587): receptor-expanded ("heter-synapse")
  matrix of shape (n * n_delay_bins, n * n_pairs); column post * n_pairs +
  pair, pair = receptor index of the synapse (neuron mode: product of the
  sorted pre and post receptor types, pre-major; connection mode: the
  synapse's own type).
* stack_hetersynapse (:839-970): per-pair dict -> stacked matrix, with the
  optional collapse of pre / post / all receptor distinctions.
* expand_conn_for_delays (:973-1027): row pre * n_delay_bins + bin,
  bin = clip(delay, 0, n_delay_bins - 1).  The fused engine decodes the bin
  of each stored edge from this row index.

The receptor split is one stable sort of the entries by pair index instead
of one table filter per receptor pair, so the cost is O(nnz log nnz) whatever
the number of receptor types.  Entry order is the reference's: pair-major,
then the order of the source matrix -- it matters because delays are
attached to entries by position (the reference attaches the delays of the
(pre, post)-sorted aggregated table to the receptor-ordered entries; that
pairing is kept as is so that the matrices are identical).
"""

from __future__ import annotations

import warnings
from collections import OrderedDict
from typing import Literal

import numpy as np
import pandas as pd
import scipy.sparse


def expand_conn_for_delays(conn, delays: np.ndarray, n_delay_bins: int = 5):
    delays = np.asarray(delays)
    if np.any(delays < 0):
        raise ValueError("delays must be non-negative")
    c = conn.tocoo()
    n_pre, n_post = c.shape
    bins = np.clip(delays, 0, n_delay_bins - 1).astype(int)
    return scipy.sparse.coo_array((c.data, (c.row * n_delay_bins + bins, c.col)),
                                  shape=(n_pre * n_delay_bins, n_post))


def _aggregate(connections: pd.DataFrame, agg: dict) -> pd.DataFrame:
    """Duplicate (pre, post) pairs merged (connections between the same
    neurons in different neuropils), sorted by (pre, post)."""
    return connections.groupby(["pre_simple_id", "post_simple_id"], as_index=False).agg(agg)


def make_sparse_mat(connections: pd.DataFrame, shape, field: str = "syn_count") -> scipy.sparse.sparray:
    """(pre, post) COO of `field` summed over duplicate pairs
    (connection.py:15-39)."""
    tab = _aggregate(connections[[field, "pre_simple_id", "post_simple_id"]], {field: "sum"})
    pre = tab["pre_simple_id"].to_numpy(dtype=int)
    post = tab["post_simple_id"].to_numpy(dtype=int)
    return scipy.sparse.coo_array((tab[field].to_numpy().reshape(-1), (pre, post)), shape=shape)


def _stacked(data, row, col, pair, n_pairs, shape):
    """Entries regrouped pair-major (stable), column post * n_pairs + pair."""
    order = np.argsort(pair, kind="stable")
    return scipy.sparse.coo_array(
        (data[order], (row[order], col[order] * n_pairs + pair[order])),
        shape=(shape[0], shape[1] * n_pairs))


def _per_pair(data, row, col, pair, keys, shape):
    """OrderedDict key -> (pre, post) COO of that pair's entries, non-empty
    pairs only, in pair order."""
    out = OrderedDict()
    order = np.argsort(pair, kind="stable")
    bounds = np.searchsorted(pair[order], np.arange(len(keys) + 1))
    for i, key in enumerate(keys):
        sel = order[bounds[i]:bounds[i + 1]]
        if len(sel):
            out[key] = scipy.sparse.coo_array((data[sel], (row[sel], col[sel])), shape=shape)
    return out


def _neuron_types(neurons: pd.DataFrame, receptor_type_col: str, dropna: str, n_ids: int):
    """Receptor-type code of every simple id (-1: no type) and the sorted type
    labels, after the NaN policy (connection.py:430-475)."""
    col = neurons[receptor_type_col]
    nan_mask = col.isna().to_numpy()
    if nan_mask.any():
        if dropna == "error":
            raise ValueError(
                f"NaN receptor types found for neurons: {neurons[nan_mask]['simple_id'].tolist()}. "
                "Set dropna='filter' to remove connections involving them, "
                "or dropna='unknown' to treat NaN as a separate receptor type.")
        if dropna == "unknown":
            col = col.astype(object).where(~nan_mask, "unknown")
            warnings.warn(f"Treating {int(nan_mask.sum())} neurons with NaN receptor types as 'unknown' receptor type")
        elif dropna != "filter":
            raise ValueError(f"dropna must be 'error', 'filter', or 'unknown', got {dropna}")
    codes, labels = pd.factorize(col, sort=True)  # NaN -> -1
    ids = neurons["simple_id"].to_numpy()
    size = max(n_ids, int(ids.max()) + 1 if len(ids) else 0)
    code_of = np.full(size, -1, np.int64)
    code_of[ids.astype(np.int64)] = codes
    return code_of, list(labels), (ids[nan_mask] if dropna == "filter" else None)


def _neuron_mode(neurons, conn, receptor_type_col, return_dict, dropna, ignore_post_type):
    """Sparse-matrix input, receptor types per neuron (connection.py:417-584)."""
    conn = conn.tocoo()
    if np.isnan(conn.data).any():
        raise ValueError("NaN values detected in connection matrix data")
    shape = conn.shape
    row = np.asarray(conn.row, np.int64)
    col = np.asarray(conn.col, np.int64)
    data = np.asarray(conn.data)
    code_of, labels, nan_ids = _neuron_types(neurons, receptor_type_col, dropna, max(shape))
    keep = np.ones(len(row), bool)
    if nan_ids is not None:
        keep = ~(np.isin(row, nan_ids) | np.isin(col, nan_ids))
        if not keep.all():
            warnings.warn(f"Filtered out {int((~keep).sum())} connections involving {len(set(nan_ids.tolist()))} "
                          "neurons with NaN receptor types")
    # a synapse is listed under the pair of its neurons' types; with
    # ignore_post_type only the presynaptic type is needed
    pre_t, post_t = code_of[row], code_of[col]
    keep &= pre_t >= 0
    if not ignore_post_type:
        keep &= post_t >= 0
    row, col, data, pre_t, post_t = row[keep], col[keep], data[keep], pre_t[keep], post_t[keep]
    n_t = len(labels)
    if ignore_post_type:
        pair = pre_t
        keys = list(labels)
        index = pd.DataFrame(list(enumerate(labels)), columns=["receptor_index", "receptor_type"])
    else:
        pair = pre_t * n_t + post_t
        keys = [(a, b) for a in labels for b in labels]
        index = pd.DataFrame([(i, a, b) for i, (a, b) in enumerate(keys)],
                             columns=["receptor_index", "pre_receptor_type", "post_receptor_type"])
    if return_dict:
        return _per_pair(data, row, col, pair, keys, shape), index
    return _stacked(data, row, col, pair, len(keys), shape), index


def make_hetersynapse_conn(
    neurons: pd.DataFrame,
    connections,
    receptor_type_col: str | None = "EI",
    receptor_type_mode: Literal["neuron", "connection"] = "neuron",
    return_dict: bool = False,
    dropna: Literal["error", "filter", "unknown"] = "error",
    ignore_post_type: bool = False,
    delay_col: str | None = None,
    n_delay_bins: int = 5,
):
    """Receptor-expanded connectivity (connection.py:218-587).

    Returns (matrix, receptor_type_index) -- or (OrderedDict pair -> (n, n)
    COO, receptor_type_index) with return_dict.  Matrix shape
    (n, n * n_pairs), or (n * n_delay_bins, n * n_pairs) with `delay_col`
    (DataFrame input only; delays in steps, aggregated as the mean over
    duplicate (pre, post) pairs and truncated to int).  With
    receptor_type_col=None only the delay expansion is done and the index
    has one row per neuron."""
    if delay_col is not None and not isinstance(connections, pd.DataFrame):
        raise ValueError("delay_col can only be used with DataFrame connections")
    n = len(neurons)

    if receptor_type_col is None:  # delays only (connection.py:297-321)
        if not isinstance(connections, pd.DataFrame):
            raise ValueError("receptor_type_col=None only supported with DataFrame connections")
        if delay_col is None:
            raise ValueError("Must provide either receptor_type_col or delay_col (or both)")
        mat = make_sparse_mat(connections, (n, n))
        delays = _aggregate(connections, {"syn_count": "sum", delay_col: "mean"})[delay_col].to_numpy().astype(int)
        index = pd.DataFrame({"simple_id": range(n)})
        if n_delay_bins > 1:
            mat = expand_conn_for_delays(mat, delays, n_delay_bins)
            index["delay_index"] = 0
        return mat, index

    if isinstance(connections, pd.DataFrame):
        delays = None
        if delay_col is not None:
            if delay_col not in connections.columns:
                raise KeyError(f"delay_col '{delay_col}' not found in connections DataFrame")
            delays = connections[delay_col].to_numpy().astype(int)
        expand = delays is not None and n_delay_bins > 1

        if receptor_type_mode == "neuron":  # (connection.py:334-357)
            if delays is not None:
                tab = _aggregate(connections, {"syn_count": "sum", delay_col: "mean"})
                mat = make_sparse_mat(tab, (n, n))
                delays = tab[delay_col].to_numpy().astype(int)
            else:
                mat = make_sparse_mat(connections, (n, n))
            out, index = _neuron_mode(neurons, mat, receptor_type_col, return_dict, dropna, ignore_post_type)
            if expand:
                out = expand_conn_for_delays(out, delays, n_delay_bins)
            return out, index

        # connection mode: the receptor type is a column of the connection
        # table (connection.py:359-415)
        shape = (n, n)
        groups = OrderedDict((k, make_sparse_mat(g, shape))
                             for k, g in connections.groupby(receptor_type_col, sort=True))
        index = pd.DataFrame(list(enumerate(groups.keys())), columns=["receptor_index", "receptor_type"])
        if return_dict:
            if expand:
                groups = OrderedDict((k, expand_conn_for_delays(v, delays, n_delay_bins)) for k, v in groups.items())
            return groups, index
        n_types = len(groups)
        mats = list(groups.values())
        out = scipy.sparse.coo_array(
            (np.concatenate([m.data for m in mats]) if mats else np.zeros(0),
             (np.concatenate([m.row for m in mats]) if mats else np.zeros(0, np.int64),
              np.concatenate([m.col * n_types + i for i, m in enumerate(mats)]) if mats else np.zeros(0, np.int64))),
            shape=(n, n * n_types))
        if expand:
            out = expand_conn_for_delays(out, delays, n_delay_bins)
        return out, index

    if isinstance(connections, scipy.sparse.sparray):
        if receptor_type_mode != "neuron":
            raise ValueError("receptor_type_mode='connection' needs a DataFrame of connections")
        return _neuron_mode(neurons, connections, receptor_type_col, return_dict, dropna, ignore_post_type)
    raise ValueError("connections must be a DataFrame or a scipy.sparse.sparray")


def stack_hetersynapse(conn_dict: dict, receptor_type_index: pd.DataFrame,
                       ignore_receptor_type: Literal["pre", "post", "all"] | None = None):
    """Per-pair matrices -> stacked (n, n * n_pairs) matrix, the inverse of
    make_hetersynapse_conn(return_dict=True) (connection.py:839-970).

    ignore_receptor_type collapses receptor distinctions and then also
    returns the reduced receptor_type_index: "post" / "pre" sum the pairs
    sharing a pre / post type (neuron mode), "all" sums every pair into one
    channel; in connection mode all three mean "all"."""
    if not conn_dict:
        raise ValueError("conn_dict is empty")
    n = next(iter(conn_dict.values())).shape[0]
    cols = set(receptor_type_index.columns)
    neuron_mode = {"pre_receptor_type", "post_receptor_type"} <= cols
    connection_mode = "receptor_type" in cols and not neuron_mode

    def stack(items, lookup, n_pairs):
        rows, cs, vals = [], [], []
        for key, mat in items:
            if key not in lookup:
                raise KeyError(f"Receptor key {key} missing from receptor_type_index")
            m = mat.tocoo()
            rows.append(m.row)
            cs.append(m.col * n_pairs + lookup[key])
            vals.append(m.data)
        return scipy.sparse.coo_array((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cs))),
                                      shape=(n, n * n_pairs))

    def relabel(labels):
        index = pd.DataFrame(list(enumerate(labels)), columns=["receptor_index", "receptor_type"])
        return index, {lab: i for i, lab in enumerate(labels)}

    if ignore_receptor_type in ("pre", "post", "all"):
        if connection_mode or ignore_receptor_type == "all":
            total = None
            for m in conn_dict.values():
                total = m.copy() if total is None else total + m
            return total.tocoo(), pd.DataFrame([(0, "all")], columns=["receptor_index", "receptor_type"])
        keep = 0 if ignore_receptor_type == "post" else 1  # the type that survives
        merged = OrderedDict()
        for key, m in conn_dict.items():
            k = key[keep]
            merged[k] = m.copy() if k not in merged else merged[k] + m
        index, lookup = relabel(list(merged.keys()))
        return stack(merged.items(), lookup, len(merged)), index

    if neuron_mode:
        lookup = {(r.pre_receptor_type, r.post_receptor_type): r.receptor_index
                  for r in receptor_type_index.itertuples(index=False)}
    elif connection_mode:
        lookup = {r.receptor_type: r.receptor_index for r in receptor_type_index.itertuples(index=False)}
    else:
        raise ValueError("receptor_type_index must contain either (pre_receptor_type, post_receptor_type) "
                         "or receptor_type columns")
    return stack(conn_dict.items(), lookup, len(receptor_type_index))


def _cell_type_codes(neurons: pd.DataFrame, cell_type_col: str, nan_in_same_group: bool):
    """root_id -> integer cell-type code lookup (connection.py:118-130).

    Every neuron whose cell type is missing gets a type of its own
    ("__none_<i>__", i counting the missing ones in table order) unless
    nan_in_same_group; the missing types that remain (and root ids absent
    from the table) share one extra code.  A duplicated root id takes the
    type of its last row.  Returns (sorted unique root ids, their codes,
    the code of a missing type)."""
    ct = neurons[cell_type_col]
    missing = ct.isna().to_numpy()
    if not nan_in_same_group and missing.any():
        ct = ct.astype(object).copy()
        ct[missing] = [f"__none_{i}__" for i in range(int(missing.sum()))]
    codes, labels = pd.factorize(ct)  # missing -> -1
    na_code = len(labels)
    codes = np.where(codes < 0, na_code, codes).astype(np.int64)
    roots = neurons["root_id"].to_numpy()
    last = ~pd.Index(roots).duplicated(keep="last")
    roots, codes = roots[last], codes[last]
    order = np.argsort(roots, kind="stable")
    return roots[order], codes[order], na_code


def _lookup(keys, values, query, default):
    """values[keys == q] for each q (keys sorted and unique), else default."""
    query = np.asarray(query)
    if len(keys) == 0:
        return np.full(len(query), default, np.int64)
    pos = np.clip(np.searchsorted(keys, query), 0, len(keys) - 1)
    return np.where(keys[pos] == query, values[pos], default)


def _pair_cell_codes(neurons, connections, cell_type_col, nan_in_same_group):
    """The first row of every distinct (pre, post) simple-id pair
    (connection.py:132-139) with its pre and post cell-type codes."""
    first = ~connections.duplicated(subset=["pre_simple_id", "post_simple_id"]).to_numpy()
    tab = connections.loc[first]
    roots, codes, na_code = _cell_type_codes(neurons, cell_type_col, nan_in_same_group)
    pre_ct = _lookup(roots, codes, tab["pre_root_id"].to_numpy(), na_code)
    post_ct = _lookup(roots, codes, tab["post_root_id"].to_numpy(), na_code)
    return (tab["pre_simple_id"].to_numpy(dtype=np.int64), tab["post_simple_id"].to_numpy(dtype=np.int64),
            pre_ct, post_ct, na_code)


def _first_seen_ids(*cols):
    """1-based ids of the distinct rows of the integer columns `cols`,
    numbered in order of first appearance (pd.factorize order)."""
    if len(cols[0]) == 0:
        return np.zeros(0, np.int64)
    key = np.stack([np.asarray(c, np.int64) for c in cols], axis=1)
    _, first, inverse = np.unique(key, axis=0, return_index=True, return_inverse=True)
    rank = np.empty(len(first), np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(first))
    return rank[inverse.reshape(-1)] + 1


def make_constraint_by_neuron_type(neurons: pd.DataFrame, connections: pd.DataFrame,
                                   nan_in_same_group: bool = True) -> scipy.sparse.sparray:
    """(n, n) COO whose value at each connected (pre, post) pair is a 1-based
    group id, one per distinct (pre cell type, post cell type) pair, numbered
    in order of first appearance in the connection table
    (connection.py:96-158).  Duplicate (pre, post) rows count once (first
    row); entries follow the table's order.  Missing cell types form one
    group with each other (nan_in_same_group) or one type per neuron."""
    pre, post, pre_ct, post_ct, _ = _pair_cell_codes(neurons, connections, "cell_type", nan_in_same_group)
    gid = _first_seen_ids(pre_ct, post_ct)
    n = neurons.shape[0]
    return scipy.sparse.coo_array((gid, (pre, post)), shape=(n, n))


def make_hetersynapse_constraint(
    neurons: pd.DataFrame,
    connections: pd.DataFrame,
    cell_type_col: str = "cell_type",
    receptor_type_col: str = "EI",
    receptor_type_mode: Literal["neuron", "connection"] = "neuron",
    constraint_mode: Literal["full", "cell_only", "cell_and_receptor"] = "full",
    nan_in_same_group: bool = True,
    ignore_post_type: bool = False,
) -> scipy.sparse.sparray:
    """Constraint groups in the receptor-expanded space of
    make_hetersynapse_conn (connection.py:590-787).

    cell_only: the (pre, post) cell-type groups of
    make_constraint_by_neuron_type, repeated pair-major for every receptor
    index (column post * n_pairs + pair), whether or not that receptor pair
    holds the synapse.  full / cell_and_receptor: one group per distinct
    (pre cell type, post cell type, receptor key) over the entries of the
    expanded matrix, numbered in the matrix's entry order; the receptor key
    is the receptor type (connection mode or ignore_post_type), else the
    (pre, post) receptor-type pair -- for cell_and_receptor as the string
    "<pre>-<post>", so pairs whose strings coincide share a group.  The cell
    types of the first table row given `cell_type_col` are used, while
    make_constraint_by_neuron_type (cell_only) reads the column "cell_type".
    The expanded matrix is built with the default NaN policy (an error on
    missing receptor types), and any mode other than full / cell_only means
    cell_and_receptor, as in the reference (connection.py:745-779)."""
    def expanded():
        return make_hetersynapse_conn(neurons, connections, receptor_type_col, receptor_type_mode,
                                      return_dict=False, ignore_post_type=ignore_post_type)

    # the (pre, post) cell-type groups come first in every mode, as in the
    # reference (so a table without "cell_type" fails the same way)
    cell = make_constraint_by_neuron_type(neurons, connections, nan_in_same_group=nan_in_same_group).tocoo()
    if constraint_mode == "cell_only":
        _, index = expanded()
        n_pairs = len(index)
        k = np.arange(n_pairs).repeat(cell.nnz)
        return scipy.sparse.coo_array(
            (np.tile(cell.data, n_pairs), (np.tile(cell.row, n_pairs), np.tile(cell.col, n_pairs) * n_pairs + k)),
            shape=(cell.shape[0], cell.shape[1] * n_pairs))

    mat, index = expanded()
    mat = mat.tocoo()
    n_pairs = len(index)
    row = np.asarray(mat.row, np.int64)
    col = np.asarray(mat.col, np.int64)
    if row.size == 0:
        return scipy.sparse.coo_array((np.zeros(0, np.int64), (row, col)), shape=mat.shape)
    pair = col % n_pairs
    post_of = col // n_pairs
    # cell types of each entry's (pre, post) neurons, from the first table
    # row of that pair; both missing if the table has no such row
    pre, post, pre_ct, post_ct, na = _pair_cell_codes(neurons, connections, cell_type_col, nan_in_same_group)
    span = max(int(pre.max(initial=0)), int(post.max(initial=0)), int(row.max()), int(post_of.max())) + 1
    order = np.argsort(pre * span + post, kind="stable")
    e_pre = _lookup((pre * span + post)[order], pre_ct[order], row * span + post_of, na)
    e_post = _lookup((pre * span + post)[order], post_ct[order], row * span + post_of, na)

    # receptor key of every receptor index
    if "receptor_type" in index.columns:
        labels = index["receptor_type"]
    elif constraint_mode == "full":
        labels = pd.Series(list(zip(index["pre_receptor_type"], index["post_receptor_type"])), dtype=object)
    else:
        labels = index["pre_receptor_type"].astype(str) + "-" + index["post_receptor_type"].astype(str)
    rec_code = pd.factorize(labels)[0].astype(np.int64)
    at = _lookup(index["receptor_index"].to_numpy(dtype=np.int64), rec_code, pair, -1)
    gid = _first_seen_ids(e_pre, e_post, at)
    return scipy.sparse.coo_array((gid, (row, col)), shape=mat.shape)


def make_hetersynapse_constrained_conn(
    neurons: pd.DataFrame,
    connections: pd.DataFrame,
    cell_type_col: str = "cell_type",
    receptor_type_col: str = "EI",
    receptor_type_mode: Literal["neuron", "connection"] = "neuron",
    constraint_mode: Literal["full", "cell_only", "cell_and_receptor"] = "full",
    nan_in_same_group: bool = True,
    dropna: Literal["error", "filter", "unknown"] = "error",
    ignore_post_type: bool = False,
):
    """(matrix, constraint, receptor_type_index) for
    SparseConstrainedConn.from_hetersynapse (connection.py:790-836): the
    matrix of make_hetersynapse_conn with `dropna`, the groups of
    make_hetersynapse_constraint (which builds its expanded matrix with the
    default NaN policy)."""
    mat, index = make_hetersynapse_conn(neurons, connections, receptor_type_col=receptor_type_col,
                                        receptor_type_mode=receptor_type_mode, return_dict=False, dropna=dropna,
                                        ignore_post_type=ignore_post_type)
    constraint = make_hetersynapse_constraint(
        neurons, connections, cell_type_col=cell_type_col, receptor_type_col=receptor_type_col,
        receptor_type_mode=receptor_type_mode, constraint_mode=constraint_mode,
        nan_in_same_group=nan_in_same_group, ignore_post_type=ignore_post_type)
    return mat, constraint, index


__all__ = ["expand_conn_for_delays", "make_constraint_by_neuron_type", "make_hetersynapse_conn",
           "make_hetersynapse_constrained_conn", "make_hetersynapse_constraint", "make_sparse_mat",
           "stack_hetersynapse"]
