"""Module state API on the CPU (no kernels): memory reset values saved and
restored beside state_dict (the reference's
tests/models/test_mem_load_save.py:103-140 flow), per-module memory access,
SpikeHistory.get_recent (tests/models/test_history.py:101-123) and
get_sparse_matrix (tests/models/test_linear.py:424-500)."""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from btorch_b200.models import ExponentialPSC, LIF, RecurrentNN, SparseConn, SparseConstrainedConn
from btorch_b200.models.base import ResetValue
from btorch_b200.models.functional import (init_net_state, named_hidden_states, named_memory_reset_values,
                                           reset_net, set_hidden_states, set_memory_reset_values)
from btorch_b200.models.history import SpikeHistory


def _model(n=6):
    conn = SparseConn(sp.coo_array(np.eye(n, dtype=np.float32)))
    return RecurrentNN(LIF(n, tau_ref=2.0, hard_reset=True), ExponentialPSC(n, tau_syn=5.0, linear=conn))


def test_reset_values_round_trip_through_torch_save(tmp_path):
    n, B = 6, 3
    m = _model(n)
    v0 = torch.linspace(-0.5, 0.5, n)
    m.neuron.set_reset_value("v", v0)
    init_net_state(m, batch_size=B)
    assert torch.equal(m.neuron.v, v0.expand(B, n))
    rv = named_memory_reset_values(m)
    assert set(rv) == {"neuron.v", "neuron.refractory", "synapse.psc"}
    assert all(isinstance(r, ResetValue) for r in rv.values())
    with torch.no_grad():
        m.neuron.v.add_(1.0)
    torch.save({"model_state": m.state_dict(), "memories_rv": rv, "hidden_states": named_hidden_states(m)},
               tmp_path / "model.pt")

    loaded = _model(n)
    ckpt = torch.load(tmp_path / "model.pt", weights_only=False)
    loaded.load_state_dict(ckpt["model_state"])
    set_memory_reset_values(loaded, ckpt["memories_rv"])
    set_hidden_states(loaded, ckpt["hidden_states"])
    after = named_memory_reset_values(loaded)
    for k in rv:
        assert after[k].sizes == rv[k].sizes
        assert torch.allclose(torch.as_tensor(after[k].value), torch.as_tensor(rv[k].value)), k
    for k, v in named_hidden_states(m).items():
        assert torch.equal(named_hidden_states(loaded)[k], v), k
    reset_net(loaded, batch_size=B)
    assert torch.equal(loaded.neuron.v, v0.expand(B, n))


def test_set_reset_values_by_module_and_by_name():
    m = _model()
    set_memory_reset_values(m, {"neuron": {"v": 0.25}, "synapse.psc": 0.5})
    init_net_state(m, batch_size=2)
    assert torch.all(m.neuron.v == 0.25) and torch.all(m.synapse.psc == 0.5)
    assert named_memory_reset_values(m, names=["neuron"]).keys() == {"neuron.v", "neuron.refractory"}
    assert named_memory_reset_values(m, names=["self.synapse.psc"]).keys() == {"synapse.psc"}
    with pytest.raises(AssertionError):
        set_memory_reset_values(m, {"neuron": {"not_a_memory": 1.0}})
    # a memory keeps its registered sizes unless told otherwise
    with pytest.raises(ValueError, match="sizes mismatch"):
        m.neuron.set_reset_value("v", 0.0, sizes=(3,))


def test_memory_accessors():
    m = _model()
    init_net_state(m, batch_size=2)
    mem = dict(m.neuron.named_memories())
    assert set(mem) == {"v", "refractory"} and mem["v"] is m.neuron.v
    assert set(m.neuron.memories_rv) == {"v", "refractory"}
    m.neuron.set_memories_rv({"refractory": 1.0})
    reset_net(m, batch_size=2)
    assert torch.all(m.neuron.refractory == 1.0)


def test_spike_history_get_recent():
    history = SpikeHistory(n_neuron=3, max_delay_steps=5)
    history.init_state(batch_size=1, dtype=torch.float32)
    for i in range(5):
        history.update(torch.tensor([[float(i), 0.0, 0.0]]))
    recent = history.get_recent(3)
    assert [r[0, 0].item() for r in recent] == [4.0, 3.0, 2.0]
    with pytest.raises(IndexError, match="n_steps .* > max_delay"):
        history.get_recent(6)


@pytest.mark.parametrize("shape", [(3, 3), (4, 2)])
def test_get_sparse_matrix(shape):
    rng = np.random.default_rng(1)
    W = (rng.random(shape) < 0.6) * rng.integers(-3, 4, shape)
    W = W.astype(np.float32)
    m = SparseConn(sp.coo_array(W), enforce_dale=False)
    mat = m.get_sparse_matrix()
    assert mat.shape == shape and mat.layout == torch.sparse_coo
    torch.testing.assert_close(mat.to_dense(), torch.tensor(W), atol=0, rtol=0)
    mat.values().sum().backward()
    assert m.magnitude.grad is not None


def test_constrained_get_sparse_matrix():
    W = sp.coo_array(([1.0, -2.0, -3.0, 1.0], ([0, 1, 0, 1], [0, 0, 1, 1])), shape=(2, 2))
    C = sp.coo_array(([1, 2, 3, 1], ([0, 0, 1, 1], [0, 1, 0, 1])), shape=(2, 2))
    m = SparseConstrainedConn(W, C, enforce_dale=False)
    with torch.no_grad():
        m.magnitude.copy_(torch.tensor([2.0, 3.0, 5.0]))
    mat = m.get_sparse_matrix()
    assert mat.shape == (2, 2)
    torch.testing.assert_close(mat.values(), m.initial_weight * m.magnitude[m._constraint_scatter_indices])
    # W[i, j] * magnitude[C[i, j] - 1], as the reference gives
    torch.testing.assert_close(mat.to_dense(), torch.tensor([[2.0, -9.0], [-10.0, 2.0]]))
    mat.values().sum().backward()
    assert m.magnitude.grad is not None


def _module_kwargs(kw):
    out = {}
    for k, v in kw.items():
        if k == "trainable_param":
            out[k] = set(v)
        elif isinstance(v, list):
            out[k] = torch.tensor(v, dtype=torch.float32)
        else:
            out[k] = v
    return out


def _build(cls, **kw):
    from btorch_b200.models import ALIF

    if cls == "ExponentialPSC":
        return ExponentialPSC(linear=torch.nn.Identity(), **{"tau_syn": 5.0, **kw})
    return {"LIF": LIF, "ALIF": ALIF}[cls](**kw)


def test_state_dicts_interchange_with_the_reference():
    """The reference's state_dicts (tests/golden/state_dict.npz): the same
    keys, shapes and values from the same constructor arguments, and loading
    one into a module built with other values gives the reference's shapes
    (uniform values compacted to scalars, per-neuron ones kept)."""
    import json

    from tests import cases

    G = cases.load("state_dict")
    for i, (cls, kw) in enumerate(json.loads(str(G["modules"]))):
        m = _build(cls, **_module_kwargs(kw))
        sd = m.state_dict()
        keys = json.loads(str(G[f"m{i}.keys"]))
        assert sorted(sd) == sorted(keys), (cls, kw)
        for k in keys:
            np.testing.assert_array_equal(sd[k].detach().numpy(), G[f"m{i}.{k}"], err_msg=f"{cls} {k}")
            assert tuple(sd[k].shape) == G[f"m{i}.{k}"].shape
        fresh = _build(cls, n_neuron=8)
        fresh.load_state_dict({k: torch.tensor(G[f"m{i}.{k}"]) for k in keys}, strict=False)
        want = json.loads(str(G[f"m{i}.reloaded"]))
        assert {k: list(v.shape) for k, v in fresh.state_dict(keep_vars=True).items()} == want, (cls, kw)
    lif = LIF(n_neuron=8)
    lif.load_state_dict({"tau": torch.full((8,), 25.0)}, strict=False)
    assert list(lif.tau.shape) == G["uniform_tau_shape"].tolist()
    lif.load_state_dict({"tau": torch.arange(8.0) + 1}, strict=False)
    assert list(lif.tau.shape) == G["nonuniform_tau_shape"].tolist()


def _param_module(n_neuron, w, **kw):
    from btorch_b200.models.base import ParamBufferMixin

    class P(ParamBufferMixin):
        def __init__(self):
            super().__init__()
            self.n_neuron = (n_neuron,) if isinstance(n_neuron, int) else tuple(n_neuron)
            self.def_param("w", w, **kw)

    return P()


def test_param_checkpoint_policy():
    """The reference's shape policy (tests/models/test_param_buffer_mixin.py):
    extra axes are never compacted; scalar / full trainable shapes hold on
    load; a trainable scalar rejects a non-scalar checkpoint."""
    m = _param_module((2, 3), torch.ones(2, 3, 4), sizes=(2, 3, 4))
    assert m.state_dict()["w"].shape == (2, 3, 4)
    m.load_state_dict({"w": torch.tensor(5.0)})
    assert m.w.shape == (2, 3, 4) and torch.all(m.w == 5.0)
    # one value per neuron without the last axis gets a unit axis
    assert _param_module(2, torch.tensor([1.0, 2.0]), sizes=(2, 3)).w.shape == (2, 1)

    auto = _param_module(4, 20.0)
    auto.load_state_dict({"w": torch.full((4,), 20.0)})
    assert auto.w.shape == ()
    auto.load_state_dict({"w": torch.tensor([1.0, 2.0, 3.0, 4.0])})
    assert auto.w.shape == (4,)

    full = _param_module(4, 2.0, trainable_param=True, trainable_shape="full")
    assert isinstance(full.w, torch.nn.Parameter) and full.w.shape == (4,)
    full.load_state_dict({"w": torch.tensor(3.0)})
    assert full.w.shape == (4,) and torch.all(full.w == 3.0)

    with pytest.raises(ValueError, match="must be uniform"):
        _param_module(4, torch.tensor([1.0, 2.0, 3.0, 4.0]), trainable_param=True, trainable_shape="scalar")
    scalar = _param_module(4, 2.0, trainable_param=True, trainable_shape="scalar")
    assert scalar.w.shape == ()
    scalar.load_state_dict({"w": torch.tensor(3.0)})
    assert scalar.w.shape == () and scalar.w.item() == 3.0
    with pytest.raises(RuntimeError, match="non-scalar checkpoint tensor"):
        scalar.load_state_dict({"w": torch.full((4,), 3.0)})
    buf = _param_module(4, 2.0, trainable_param=False, trainable_shape="scalar")
    buf.load_state_dict({"w": torch.tensor([1.0, 2.0, 3.0, 4.0])})
    assert buf.w.shape == (4,)


def test_constraint_group_ids_must_be_positive_integers():
    W = sp.coo_array(([1.0, -2.0], ([0, 1], [0, 0])), shape=(2, 2))
    for bad in ([1, -1], [1, 1.5]):
        C = sp.coo_array((bad, ([0, 1], [0, 0])), shape=(2, 2))
        with pytest.raises(ValueError, match="group ids"):
            SparseConstrainedConn(W, C, enforce_dale=False)
