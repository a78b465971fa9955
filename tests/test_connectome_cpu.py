"""Connectome input format (btorch/connectome/connection.py): the matrices
make_hetersynapse_conn and stack_hetersynapse build equal the reference's
entry for entry -- same order, same values, same receptor index -- on the
seeded tables of tests/golden/connectome_format.npz (made by the reference),
plus the reference's own known-answer checks
(tests/connectome/test_delay_expansion.py:160-340,
tests/models/test_hetersynapse_conn.py:112-210, 536-812)."""

import io
import json
from collections import OrderedDict

import numpy as np
import pandas as pd
import pytest
import scipy.sparse

from btorch_b200.connectome import make_hetersynapse_conn, stack_hetersynapse
from tests import cases

G = cases.load("connectome_format")


def tables(t):
    neu = pd.DataFrame({k.split(".")[-1]: v for k, v in G.items() if k.startswith(f"in.{t}.neurons.")})
    con = pd.DataFrame({k.split(".")[-1]: v for k, v in G.items() if k.startswith(f"in.{t}.conns.")})
    neu["EI"] = neu["EI"].astype(object).where(neu["EI"] != "nan", np.nan)
    con["nt"] = con["nt"].astype(object)
    return neu, con


def golden_coo(name):
    return (G[f"{name}.row"], G[f"{name}.col"], G[f"{name}.data"], tuple(G[f"{name}.shape"]))


def golden_index(key):
    return pd.read_json(io.StringIO(str(G[key])), orient="split")


def assert_same(m, name):
    m = m.tocoo()
    row, col, data, shape = golden_coo(name)
    assert m.shape == shape
    np.testing.assert_array_equal(m.row, row, err_msg=name)
    np.testing.assert_array_equal(m.col, col, err_msg=name)
    np.testing.assert_array_equal(m.data, data, err_msg=name)


def assert_index(idx, key):
    want = golden_index(key)
    assert list(idx.columns) == list(want.columns)
    for c in idx.columns:
        assert [str(v) for v in idx[c]] == [str(v) for v in want[c]], (key, c)


RUNS = ["neuron", "neuron_ignore_post", "neuron_delay", "neuron_filter", "neuron_unknown",
        "neuron_filter_ignore_post", "connection", "connection_delay", "delay_only"]


@pytest.mark.parametrize("name", RUNS)
@pytest.mark.filterwarnings("ignore::UserWarning")
def test_matches_reference_fixture(name):
    kw = json.loads(str(G[f"{name}.kwargs"]))
    neu_nan, con_dup = tables("dup")
    neu_ok = neu_nan.copy()
    neu_ok.loc[neu_ok.EI.isna(), "EI"] = "E"
    neu_u, con_u = tables("uniq")
    neu, con = {"neuron_filter": (neu_nan, con_dup), "neuron_unknown": (neu_nan, con_dup),
                "neuron_filter_ignore_post": (neu_nan, con_dup),
                "connection_delay": (neu_u, con_u)}.get(name, (neu_ok, con_dup))
    m, idx = make_hetersynapse_conn(neu, con, **kw)
    assert_same(m, name)
    assert_index(idx, f"{name}.index")


@pytest.mark.parametrize("mode", ["dict_neuron", "dict_connection"])
def test_dict_and_stack_match_reference_fixture(mode):
    neu_nan, con = tables("dup")
    neu = neu_nan.copy()
    neu.loc[neu.EI.isna(), "EI"] = "E"
    kw = {} if mode == "dict_neuron" else dict(receptor_type_col="nt", receptor_type_mode="connection")
    d, idx = make_hetersynapse_conn(neu, con, return_dict=True, **kw)
    keys = [list(k) if isinstance(k, tuple) else k for k in d]
    assert keys == json.loads(str(G[f"{mode}.keys"]))
    for i, m in enumerate(d.values()):
        assert_same(m, f"{mode}.{i}")
    assert_index(idx, f"{mode}.index")
    assert_same(stack_hetersynapse(d, idx), f"{mode}.stacked")
    for how in ("pre", "post", "all"):
        m2, idx2 = stack_hetersynapse(d, idx, ignore_receptor_type=how)
        assert_same(m2, f"{mode}.collapse_{how}")
        assert_index(idx2, f"{mode}.collapse_{how}.index")


def small_tables():
    """3 neurons (E, E, I) and 4 connections with delays
    (test_delay_expansion.py:163-190)."""
    neurons = pd.DataFrame({"simple_id": [0, 1, 2], "root_id": [100, 101, 102], "EI": ["E", "E", "I"]})
    conns = pd.DataFrame({"pre_simple_id": [0, 0, 1, 2], "post_simple_id": [1, 2, 2, 0],
                          "pre_root_id": [100, 100, 101, 102], "post_root_id": [101, 102, 102, 100],
                          "syn_count": [1, 1, 1, 1], "delay_steps": [1, 2, 0, 3]})
    return neurons, conns


def test_combined_delay_and_receptor_known_answer():
    neurons, conns = small_tables()
    conn, idx = make_hetersynapse_conn(neurons, conns, receptor_type_col="EI", receptor_type_mode="neuron",
                                       delay_col="delay_steps", n_delay_bins=5)
    assert conn.shape == (15, 12)
    dense = conn.toarray()
    assert dense[1, 4] == 1 and dense[2, 9] == 1 and dense[5, 9] == 1 and dense[13, 2] == 1
    assert conn.nnz == len(conns)
    plain, idx_plain = make_hetersynapse_conn(neurons, conns, receptor_type_col="EI", receptor_type_mode="neuron")
    assert plain.shape[1] == conn.shape[1]
    pd.testing.assert_frame_equal(idx, idx_plain)


def test_delays_only_and_empty():
    neurons, conns = small_tables()
    conn, idx = make_hetersynapse_conn(neurons, conns, receptor_type_col=None, delay_col="delay_steps",
                                       n_delay_bins=5)
    assert conn.shape == (15, 3) and len(idx) == 3
    empty = conns.iloc[:0]
    conn, _ = make_hetersynapse_conn(neurons, empty, receptor_type_col=None, delay_col="delay_steps",
                                     n_delay_bins=5)
    assert conn.shape == (15, 3) and conn.nnz == 0


def test_errors():
    neurons, conns = small_tables()
    with pytest.raises(KeyError):
        make_hetersynapse_conn(neurons, conns, receptor_type_col="receptor_type", receptor_type_mode="connection",
                               delay_col="invalid_delay_col")
    with pytest.raises(ValueError, match="DataFrame"):
        make_hetersynapse_conn(neurons, scipy.sparse.coo_array((3, 3)), delay_col="delay_steps")
    with pytest.raises(ValueError, match="either receptor_type_col or delay_col"):
        make_hetersynapse_conn(neurons, conns, receptor_type_col=None)
    nan_neurons = neurons.assign(EI=["E", np.nan, "I"])
    with pytest.raises(ValueError, match="NaN receptor types found"):
        make_hetersynapse_conn(nan_neurons, conns)
    with pytest.warns(UserWarning, match="Filtered out .* connections involving"):
        m, _ = make_hetersynapse_conn(nan_neurons, conns, dropna="filter")
    assert m.shape[0] == 3 and m.nnz == 2  # 0->1 and 1->2 involve neuron 1
    with pytest.warns(UserWarning, match="Treating .* neurons with NaN receptor types"):
        _, idx = make_hetersynapse_conn(nan_neurons, conns, dropna="unknown")
    assert len(idx) == 9


def test_stack_collapse_known_values():
    """Neuron-mode collapse data (test_hetersynapse_conn.py:695-772)."""
    n = 3
    mats = OrderedDict([(("A", "X"), scipy.sparse.coo_array(([1], ([0], [1])), shape=(n, n))),
                        (("A", "Y"), scipy.sparse.coo_array(([3], ([0], [2])), shape=(n, n))),
                        (("B", "X"), scipy.sparse.coo_array(([2], ([1], [0])), shape=(n, n))),
                        (("B", "Y"), scipy.sparse.coo_array(([5], ([2], [1])), shape=(n, n)))])
    idx = pd.DataFrame([(0, "A", "X"), (1, "A", "Y"), (2, "B", "X"), (3, "B", "Y")],
                       columns=["receptor_index", "pre_receptor_type", "post_receptor_type"])
    full = stack_hetersynapse(mats, idx).toarray()
    assert full[0, 1 * 4 + 0] == 1 and full[0, 2 * 4 + 1] == 3 and full[1, 0 * 4 + 2] == 2 and full[2, 1 * 4 + 3] == 5
    post, pidx = stack_hetersynapse(mats, idx, ignore_receptor_type="post")
    assert list(pidx.receptor_type) == ["A", "B"]
    p = post.toarray()
    assert p[0, 1 * 2 + 0] == 1 and p[0, 2 * 2 + 0] == 3 and p[1, 0 * 2 + 1] == 2 and p[2, 1 * 2 + 1] == 5
    pre, qidx = stack_hetersynapse(mats, idx, ignore_receptor_type="pre")
    assert list(qidx.receptor_type) == ["X", "Y"]
    q = pre.toarray()
    assert q[0, 1 * 2 + 0] == 1 and q[0, 2 * 2 + 1] == 3 and q[1, 0 * 2 + 0] == 2 and q[2, 1 * 2 + 1] == 5
    tot, _ = stack_hetersynapse(mats, idx, ignore_receptor_type="all")
    np.testing.assert_array_equal(tot.toarray(), [[0, 1, 3], [2, 0, 0], [0, 5, 0]])
    with pytest.raises(KeyError):
        stack_hetersynapse(OrderedDict([(("Z", "Z"), mats[("A", "X")])]), idx)
