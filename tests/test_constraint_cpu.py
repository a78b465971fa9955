"""Constraint-group builders of btorch_b200.connectome against the seeded
tables of tests/golden/connectome_constraint.npz (made by the reference),
plus the reference's own property checks
(tests/models/test_hetersynapse_conn.py:212-310, 380-470) and hand-worked
cases."""

import io
import json

import numpy as np
import pandas as pd
import pytest
import scipy.sparse

from btorch_b200.connectome import (make_constraint_by_neuron_type, make_hetersynapse_conn,
                                    make_hetersynapse_constrained_conn, make_hetersynapse_constraint)
from tests import cases

G = cases.load("connectome_constraint")
N_RUNS = sum(1 for k in G if k.startswith("hetero.") and k.endswith(".kwargs"))


def tables():
    neu = pd.DataFrame({k.split(".")[-1]: v for k, v in G.items() if k.startswith("in.neurons.")})
    con = pd.DataFrame({k.split(".")[-1]: v for k, v in G.items() if k.startswith("in.conns.")})
    for c in ("cell_type", "EI", "ct2"):
        neu[c] = neu[c].astype(object).where(neu[c] != "nan", np.nan)
    con["nt"] = con["nt"].astype(object)
    return neu, con


def assert_same(m, name):
    m = m.tocoo()
    assert m.shape == tuple(G[f"{name}.shape"])
    for f in ("row", "col", "data"):
        np.testing.assert_array_equal(np.asarray(getattr(m, f)), G[f"{name}.{f}"], err_msg=f"{name}.{f}")


@pytest.mark.parametrize("nan_in_same_group", [True, False])
def test_by_neuron_type_matches_reference(nan_in_same_group):
    neu, con = tables()
    assert neu.cell_type.isna().sum() == 3
    m = make_constraint_by_neuron_type(neu, con, nan_in_same_group=nan_in_same_group)
    assert_same(m, f"by_type.{int(nan_in_same_group)}")


@pytest.mark.parametrize("i", range(N_RUNS))
def test_hetersynapse_constraint_matches_reference(i):
    neu, con = tables()
    kw = json.loads(str(G[f"hetero.{i}.kwargs"]))
    assert_same(make_hetersynapse_constraint(neu, con, **kw), f"hetero.{i}")


@pytest.mark.parametrize("mode", ["cell_only", "cell_and_receptor"])
def test_constrained_conn_and_groups_match_reference(mode):
    """The combined builder, then SparseConstrainedConn.from_hetersynapse:
    every stored nonzero lands in the reference's group."""
    from btorch_b200.models import SparseConstrainedConn

    neu, con = tables()
    m, c, idx = make_hetersynapse_constrained_conn(neu, con, constraint_mode=mode)
    assert_same(m, f"combined.{mode}.conn")
    assert_same(c, f"combined.{mode}.constraint")
    want = pd.read_json(io.StringIO(str(G[f"combined.{mode}.index"])), orient="split")
    assert list(idx.columns) == list(want.columns)
    np.testing.assert_array_equal(idx.to_numpy().astype(str), want.to_numpy().astype(str))
    lin = SparseConstrainedConn.from_hetersynapse(m.astype(np.float32), c, idx, enforce_dale=True)
    np.testing.assert_array_equal(lin._constraint_scatter_indices.numpy(), G[f"combined.{mode}.group"])
    assert lin.magnitude.numel() == int(G[f"combined.{mode}.n_groups"])
    assert lin.constraint_info["receptor_type_index"] is idx


def _toy():
    """Four neurons: types a, a, b, missing; E, I, E, E."""
    neu = pd.DataFrame({"root_id": [10, 11, 12, 13], "simple_id": [0, 1, 2, 3],
                        "cell_type": ["a", "a", "b", np.nan], "EI": ["E", "I", "E", "E"]})
    pre = [0, 1, 0, 2, 3, 0, 2, 1]
    post = [2, 2, 1, 0, 0, 2, 3, 3]
    con = pd.DataFrame({"pre_simple_id": pre, "post_simple_id": post,
                        "pre_root_id": [10 + p for p in pre], "post_root_id": [10 + q for q in post],
                        "syn_count": [1, 2, 3, 4, 5, 6, 7, 8]})
    return neu, con


def test_by_neuron_type_hand_worked():
    neu, con = _toy()
    m = make_constraint_by_neuron_type(neu, con)
    # rows in table order, the duplicate (0, 2) dropped; pairs
    # (a,b) (a,b) (a,a) (b,a) (nan,a) (b,nan) (a,nan) -> 1 1 2 3 4 5 6
    np.testing.assert_array_equal(m.row, [0, 1, 0, 2, 3, 2, 1])
    np.testing.assert_array_equal(m.col, [2, 2, 1, 0, 0, 3, 3])
    np.testing.assert_array_equal(m.data, [1, 1, 2, 3, 4, 5, 6])
    assert m.shape == (4, 4)
    # one missing neuron: its own type either way
    np.testing.assert_array_equal(make_constraint_by_neuron_type(neu, con, nan_in_same_group=False).data,
                                  m.data)


def test_missing_types_grouped_or_split():
    neu = pd.DataFrame({"root_id": [1, 2, 3], "simple_id": [0, 1, 2],
                        "cell_type": [np.nan, float("nan"), "a"], "EI": ["E", "E", "E"]})
    con = pd.DataFrame({"pre_simple_id": [0, 1, 0], "post_simple_id": [2, 2, 1], "pre_root_id": [1, 2, 1],
                        "post_root_id": [3, 3, 2], "syn_count": [1, 1, 1]})
    np.testing.assert_array_equal(make_constraint_by_neuron_type(neu, con).data, [1, 1, 2])
    np.testing.assert_array_equal(make_constraint_by_neuron_type(neu, con, nan_in_same_group=False).data, [1, 2, 3])
    # a root id missing from the neuron table reads as a missing type
    con.loc[2, "post_root_id"] = 99
    np.testing.assert_array_equal(make_constraint_by_neuron_type(neu, con).data, [1, 1, 2])


def test_hetersynapse_constraint_hand_worked():
    neu, con = _toy()
    conn, idx = make_hetersynapse_conn(neu, con)
    assert list(idx.itertuples(index=False, name=None)) == [(0, "E", "E"), (1, "E", "I"), (2, "I", "E"),
                                                            (3, "I", "I")]
    full = make_hetersynapse_constraint(neu, con, constraint_mode="full")
    assert full.shape == conn.shape
    np.testing.assert_array_equal(full.row, conn.tocoo().row)
    np.testing.assert_array_equal(full.col, conn.tocoo().col)
    # one group per (pre type, post type, pre EI, post EI), in entry order
    c = conn.tocoo()
    types = {0: "a", 1: "a", 2: "b", 3: None}
    ei = {0: "E", 1: "I", 2: "E", 3: "E"}
    keys = [(types[r], types[k // 4], ei[r], ei[k // 4]) for r, k in zip(c.row, c.col)]
    want = pd.factorize(pd.Series(keys, dtype=object))[0] + 1
    np.testing.assert_array_equal(full.data, want)
    # cell_only: the cell-type groups repeated for each of the four pairs
    cell = make_constraint_by_neuron_type(neu, con)
    only = make_hetersynapse_constraint(neu, con, constraint_mode="cell_only")
    assert only.shape == conn.shape and only.nnz == 4 * cell.nnz
    np.testing.assert_array_equal(only.data, np.tile(cell.data, 4))
    np.testing.assert_array_equal(only.col, np.concatenate([cell.col * 4 + k for k in range(4)]))


def test_reference_property_checks():
    """The reference's checks on its own generated tables: shapes agree with
    the matrix, ids start at 1, cell_only never has more groups than full."""
    rng = np.random.default_rng(42)
    n = 60
    neu = pd.DataFrame({"root_id": np.arange(1000, 1000 + n), "simple_id": np.arange(n),
                        "cell_type": [f"type_{i % 5}" for i in range(n)],
                        "EI": rng.choice(["E", "I"], size=n, p=[0.7, 0.3])})
    k = int(n * n * 0.15)
    pre, post = rng.integers(0, n, k), rng.integers(0, n, k)
    keep = pre != post
    con = pd.DataFrame({"pre_simple_id": pre[keep], "post_simple_id": post[keep],
                        "syn_count": rng.integers(1, 10, keep.sum())})
    con["pre_root_id"] = con.pre_simple_id + 1000
    con["post_root_id"] = con.post_simple_id + 1000
    groups = {}
    for mode in ("full", "cell_only", "cell_and_receptor"):
        conn, c, idx = make_hetersynapse_constrained_conn(neu, con, constraint_mode=mode)
        assert scipy.sparse.issparse(c) and c.nnz > 0
        assert c.shape == conn.shape and c.data.min() >= 1
        groups[mode] = int(c.data.max())
    assert groups["cell_only"] <= 25 <= groups["full"]
    assert groups["full"] == groups["cell_and_receptor"]  # E/I pairs: the same key either way


def test_error_behaviour():
    neu, con = _toy()
    # an unknown mode is cell_and_receptor (no error), as in the reference
    np.testing.assert_array_equal(make_hetersynapse_constraint(neu, con, constraint_mode="neither").data,
                                  make_hetersynapse_constraint(neu, con, constraint_mode="cell_and_receptor").data)
    # the constraint's expanded matrix keeps the default NaN policy, even
    # when the combined call asks to filter
    neu.loc[1, "EI"] = np.nan
    with pytest.raises(ValueError, match="NaN receptor types"):
        make_hetersynapse_constrained_conn(neu, con, dropna="filter")
    # cell types are always read from "cell_type" first
    with pytest.raises(KeyError):
        make_hetersynapse_constraint(neu.rename(columns={"cell_type": "ct"}), con, cell_type_col="ct")


def test_empty_connection_table():
    """An empty table gives empty constraint matrices of the full shape, as
    in the reference."""
    neu, con = _toy()
    con = con.iloc[:0]
    assert make_constraint_by_neuron_type(neu, con).shape == (4, 4)
    for mode in ("full", "cell_only", "cell_and_receptor"):
        c = make_hetersynapse_constraint(neu, con, constraint_mode=mode)
        assert c.shape == (4, 16) and c.nnz == 0


@pytest.mark.parametrize("mode", ["cell_only", "cell_and_receptor"])
def test_group_helpers_match_reference(mode):
    """get_group_info / set_group_magnitude (by group and by receptor pair) /
    get_weights_by_group as the reference's (linear.py:763-867)."""
    import torch

    from btorch_b200.models import SparseConstrainedConn

    neu, con = tables()
    m, c, idx = make_hetersynapse_constrained_conn(neu, con, constraint_mode=mode)
    lin = SparseConstrainedConn.from_hetersynapse(m.astype(np.float32), c, idx, enforce_dale=True)
    with torch.no_grad():
        lin.magnitude.copy_(torch.linspace(0.5, 1.5, lin.magnitude.numel()))
    lin.set_group_magnitude(group_id=1, value=2.5)
    lin.set_group_magnitude(receptor_pair=("E", "I"), value=0.25)
    got = lin.get_group_info(include_weights=True)
    want = pd.read_json(io.StringIO(str(G[f"combined.{mode}.group_info"])), orient="split")
    assert list(got.columns) == list(want.columns)
    for col in got.columns:
        if got[col].dtype.kind in "iu" or want[col].dtype.kind in "iu":
            np.testing.assert_array_equal(got[col].to_numpy(), want[col].to_numpy(), err_msg=col)
        elif got[col].dtype.kind == "f":
            np.testing.assert_allclose(got[col].to_numpy(), want[col].to_numpy(), rtol=1e-6, err_msg=col)
        else:
            np.testing.assert_array_equal(got[col].astype(str).to_numpy(), want[col].astype(str).to_numpy())
    wbg = lin.get_weights_by_group()
    np.testing.assert_array_equal([len(wbg[g]) for g in sorted(wbg)], G[f"combined.{mode}.by_group_len"])
    np.testing.assert_array_equal(np.concatenate([wbg[g].detach().numpy() for g in sorted(wbg)]),
                                  G[f"combined.{mode}.by_group"])
    with pytest.raises(ValueError, match="Exactly one"):
        lin.set_group_magnitude()
    with pytest.raises(ValueError, match="Exactly one"):
        lin.set_group_magnitude(group_id=0, receptor_pair=("E", "E"))
