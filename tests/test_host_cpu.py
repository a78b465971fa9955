"""Host-side logic that needs no GPU: the C-ABI library loads and exports every
declared symbol, the layout builder, config registry, module state API."""

import re
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from btorch_b200 import _lib as L
from btorch_b200 import config
from btorch_b200._sparse_config import SparseConfigRegistry, TritonSparseConfig
from btorch_b200.connectome import expand_conn_for_delays
from btorch_b200.models import LIF, ALIF, ExponentialPSC, RecurrentNN, SparseConn
from btorch_b200.models._ops import build_layout
from btorch_b200.models.functional import init_net_state, named_hidden_states, prepare_sparse_modules, reset_net

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "btorch_b200.h").read_text()
    return sorted(set(re.findall(r"BT_API\s+(?:const\s+char\*|int64_t|int)\s+(bt_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    syms = declared_symbols()
    assert len(syms) >= 16
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(L.exported_symbols())
    assert lib.bt_abi_version() == L.ABI_VERSION == 11


def test_layout_matches_numpy_reference():
    rng = np.random.default_rng(0)
    n_pre, n_post, D = 37, 29, 4
    dense = (rng.random((n_pre * D, n_post)) < 0.2) * rng.standard_normal((n_pre * D, n_post))
    c = sp.coo_array(dense.astype(np.float32)).T
    c.sum_duplicates()
    idx = torch.tensor(np.stack([c.row, c.col]), dtype=torch.long)
    lay = build_layout(idx, n_pre, n_post, D)
    post, src = c.row, c.col
    # CSC: canonical order, pre|bin packing
    assert np.array_equal(lay.csc_ptr.numpy(), np.concatenate([[0], np.cumsum(np.bincount(post, minlength=n_post))]))
    packed = lay.csc_src.numpy().view(np.uint32)
    assert np.array_equal(packed & ((1 << 25) - 1), src // D)
    assert np.array_equal(packed >> 25, src % D)
    # CSR: grouped by pre, canonical order inside, perm maps back
    perm = lay.csr_perm.numpy()
    assert sorted(perm.tolist()) == list(range(c.nnz))
    pre_of = src[perm] // D
    assert np.all(np.diff(pre_of) >= 0)
    for j in range(n_pre):
        seg = perm[lay.csr_ptr[j]: lay.csr_ptr[j + 1]]
        assert np.all(np.diff(seg) > 0)
    dst = lay.csr_dst.numpy().view(np.uint32)[: c.nnz]
    assert np.array_equal(dst & ((1 << 25) - 1), post[perm])
    assert np.array_equal(dst >> 25, (src % D)[perm])
    assert lay.csr_dst.numel() % 4 == 0


def test_layout_rejects_non_canonical_order():
    idx = torch.tensor([[1, 0], [0, 0]], dtype=torch.long)
    with pytest.raises(ValueError, match="canonical"):
        build_layout(idx, 2, 2, 1)
    with pytest.raises(ValueError, match="outside"):
        build_layout(torch.tensor([[0], [5]]), 2, 2, 1)


def test_sparse_config_registry_semantics():
    reg = SparseConfigRegistry()
    tpl = reg.backend("triton")
    assert isinstance(tpl, TritonSparseConfig)
    r = reg.resolve("triton", {"hash": False, "direction": "scatter"})
    assert tpl.hash is True and r.hash is False and r.direction == "scatter"
    with pytest.raises(ValueError):
        reg.resolve("b200", {"no_such_field": 1})
    with pytest.raises(ValueError):
        reg.resolve("triton", {"edge_block": 3})
    with pytest.raises(ValueError):
        reg.backend("cusparse")
    with pytest.raises(ValueError):
        reg.resolve("b200", {"direction": "sideways"})
    # the process-wide registry modules resolve against (btorch.config.sparse)
    assert isinstance(config.sparse, SparseConfigRegistry)
    assert isinstance(config.sparse.backend("triton"), TritonSparseConfig)


def test_sparseconn_state_dict_and_prepare_scope():
    W = sp.coo_array(np.array([[1.0, 0.0], [0.0, 2.0]], np.float32))
    m = SparseConn(W, enforce_dale=False, sparse_backend="native")
    assert sorted(m.state_dict()) == ["indices", "magnitude"]
    W2 = sp.coo_array(np.array([[0.0, 3.0], [4.0, 0.0]], np.float32))
    t = SparseConn(W2, enforce_dale=False)
    t.load_state_dict(m.state_dict())
    assert torch.equal(t.indices, m.indices)
    lay = t.layout()
    assert lay.csc_ptr.tolist() == [0, 1, 2]
    with pytest.raises(RuntimeError):
        t.finish_sparse()
    with prepare_sparse_modules(t):
        assert t._sparse_prepare_depth == 1
    assert t._sparse_prepare_depth == 0


def test_sparseconn_has_no_cpu_path():
    m = SparseConn(sp.coo_array(np.eye(3, dtype=np.float32)))
    with pytest.raises(RuntimeError, match="CUDA"):
        m(torch.ones(3))
    # a width other than in_features is refused before any kernel sees it
    for bad in (torch.ones(2), torch.ones(4, 5)):
        with pytest.raises(RuntimeError, match="takes 3 input features"):
            m(bad)


def test_memory_module_reset_inplace_and_state_names():
    n = 8
    rnn = RecurrentNN(LIF(n, tau_ref=2.0), ExponentialPSC(n, 5.0, SparseConn(sp.coo_array(np.eye(n, dtype=np.float32)))))
    init_net_state(rnn, batch_size=2, dtype=torch.float32)
    v = rnn.neuron.v
    v.fill_(3.0)
    reset_net(rnn, inplace=True)
    assert rnn.neuron.v is v and float(v.abs().sum()) == 0.0
    assert sorted(named_hidden_states(rnn)) == ["neuron.refractory", "neuron.v", "synapse.psc"]
    with pytest.raises(ValueError):
        reset_net(rnn, batch_size=3, inplace=True)
    a = ALIF(n, g_k_init=0.5)
    init_net_state(a, batch_size=(2, 3), dtype=torch.float32)
    assert a.g_k.shape == (2, 3, n) and float(a.g_k[0, 0, 0]) == 0.5


def test_expand_conn_for_delays_rows():
    conn = sp.coo_array(([1.0, 2.0], ([0, 1], [1, 2])), shape=(3, 3))
    d = expand_conn_for_delays(conn, np.array([1, 3]), n_delay_bins=5)
    assert d.shape == (15, 3)
    dense = d.toarray()
    assert dense[0 * 5 + 1, 1] == 1.0 and dense[1 * 5 + 3, 2] == 2.0
    with pytest.raises(ValueError):
        expand_conn_for_delays(conn, np.array([-1, 0]))


def test_engine_plan_matching_on_cpu_modules():
    n = 16
    conn = SparseConn(sp.coo_array(np.eye(n, dtype=np.float32)))
    rnn = RecurrentNN(LIF(n, tau_ref=2.0, hard_reset=True), ExponentialPSC(n, 5.0, conn))
    plan, why = rnn.fused_plan()
    assert plan is not None, why
    assert set(plan.paths.values()) == {"v", "ref", "psc"}
    rnn2 = RecurrentNN(LIF(n), ExponentialPSC(n, 5.0, torch.nn.Linear(n, n)))
    plan2, why2 = rnn2.fused_plan()
    assert plan2 is None and "SparseConn" in why2


def test_empty_connection_runs_per_module():
    """A connection without synapses (valid in the reference) is declined by
    the fused engine and the fused BPTT, so the per-module kernels run it;
    its layout keeps non-null padded CSR arrays."""
    from btorch_b200.models import bptt

    n = 16
    conn = SparseConn(sp.coo_array((n, n), dtype=np.float32))
    rnn = RecurrentNN(LIF(n, tau_ref=2.0, hard_reset=True), ExponentialPSC(n, 5.0, conn))
    plan, why = rnn.fused_plan()
    assert plan is None and "no synapses" in why
    paths, why = bptt.match(rnn)
    assert paths is None and "no synapses" in why
    lay = build_layout(conn.indices, n, n)
    assert lay.nnz == 0 and lay.csr_dst.numel() == 4
    assert np.array_equal(lay.csc_ptr.numpy(), np.zeros(n + 1)) and np.array_equal(lay.csr_ptr.numpy(), np.zeros(n + 1))


def test_neuron_desc_cache_follows_parameter_changes():
    """The per-module path's neuron descriptor is cached on the module and
    rebuilt when a parameter is modified in place, rebound, or dt changes."""
    import torch

    from btorch_b200.models import ALIF, LIF
    from btorch_b200.models._ops import neuron_desc

    for cls in (LIF, ALIF):
        m = cls(8, v_threshold=1.0, tau_ref=2.0)
        d1, _ = neuron_desc(m, 1.0)
        d2, _ = neuron_desc(m, 1.0)
        assert d1 is d2
        assert neuron_desc(m, 0.5)[0] is not d1
        d3, _ = neuron_desc(m, 1.0)
        with torch.no_grad():
            m.v_threshold.fill_(2.0)
        d4, _ = neuron_desc(m, 1.0)
        assert d4 is not d3 and d4.sv[0] == 2.0
        m.v_threshold = torch.tensor(3.0)
        d5, _ = neuron_desc(m, 1.0)
        assert d5 is not d4 and d5.sv[0] == 3.0


def test_fused_bptt_match_rules():
    """Which models the fused BPTT takes (host logic only): LIF/ALIF +
    ExponentialPSC over a square SparseConn, optional nn.Linear input, state
    stacks of v / psc / g_k / refractory; everything else steps module by
    module."""
    import numpy as np
    import scipy.sparse as sp

    from btorch_b200.models import ALIF, LIF, DelayedPSC, DenseConn, ExponentialPSC, RecurrentNN, SparseConn
    from btorch_b200.models import bptt

    n = 16
    W = sp.coo_array(sp.random(n, n, density=0.2, random_state=0, dtype=np.float32))

    def net(neuron=None, syn=None, **kw):
        neuron = neuron or LIF(n, tau_ref=2.0)
        syn = syn or ExponentialPSC(n, 5.0, SparseConn(W))
        return RecurrentNN(neuron, syn, **kw)

    paths, why = bptt.match(net())
    assert why == "" and set(paths.values()) == {"v", "ref", "psc"}
    paths, _ = bptt.match(net(ALIF(n), update_state_names=("neuron.g_k",)))
    assert paths == {"neuron.g_k": "gk"}
    assert bptt.match(net(neuron_inp_module=DenseConn(4, n)))[0] is not None
    assert bptt.match(net(syn=DelayedPSC(ExponentialPSC(n, 5.0, SparseConn(W)), max_delay_steps=3)))[1] == "synapse"
    assert bptt.match(net(cpu_offload=True))[0] is None
    rect = sp.coo_array(sp.random(n, 2 * n, density=0.2, random_state=1, dtype=np.float32))
    assert bptt.match(net(syn=ExponentialPSC(n, 5.0, SparseConn(rect))))[0] is None


def test_engine_checks_the_input_shape_before_any_device_work():
    """With an input layer, x must be [T, *batch, in_features] for the
    network's batch: a wider row would index past the projection weights."""
    from btorch_b200.models import DenseConn
    from btorch_b200.models import engine

    n = 16
    rnn = RecurrentNN(LIF(n), ExponentialPSC(n, 5.0, SparseConn(sp.coo_array(np.eye(n, dtype=np.float32)))),
                      neuron_inp_module=DenseConn(4, n))
    init_net_state(rnn, batch_size=3)
    plan, _ = rnn.fused_plan()
    with pytest.raises(RuntimeError, match="takes 4 channels"):
        engine.run(plan, rnn, torch.zeros(5, 3, 5))
    with pytest.raises(RuntimeError, match="batch"):
        engine.run(plan, rnn, torch.zeros(5, 6, 4))
    with pytest.raises(RuntimeError, match="CUDA"):  # a well-formed input gets as far as the device check
        engine.run(plan, rnn, torch.zeros(5, 3, 4))


def test_psc_time_constants_must_be_scalar_or_per_neuron():
    """The kernels read one time constant per neuron: other lengths are refused
    on the host (the reference's broadcast against psc raises for them)."""
    for tau in (5.0, torch.full((8,), 5.0)):
        coef, t = ExponentialPSC(8, tau_syn=tau, linear=torch.nn.Identity()).coefficients(1.0)
        assert coef.numel() == t.numel() in (1, 8)
    with pytest.raises(RuntimeError, match="expected 1 or 8"):
        ExponentialPSC(8, tau_syn=torch.full((3,), 5.0), linear=torch.nn.Identity()).coefficients(1.0)


def test_weight_length_must_match_the_stored_nonzeros():
    m = SparseConn(sp.coo_array(np.eye(4, dtype=np.float32)), enforce_dale=False)
    assert m._edge_weight().numel() == 4
    m.magnitude = torch.nn.Parameter(torch.ones(3))
    with pytest.raises(RuntimeError, match="4 stored nonzeros but 3 weights"):
        m._edge_weight()
    with pytest.raises(RuntimeError, match="4 stored nonzeros but 3 weights"):
        m(torch.ones(2, 4))


def test_neuron_parameters_reach_the_kernels_per_neuron():
    """A parameter narrower than the neuron shape (one value per column of a
    2-D population) is broadcast to one value per neuron before the kernels
    read it; per-sample parameters, which the kernels cannot express, are
    refused instead of being read past their end."""
    from btorch_b200.models._ops import _build_neuron_desc

    lif = LIF((4, 5), tau=torch.tensor([10.0, 20.0, 30.0, 40.0, 50.0]))
    _, keep = _build_neuron_desc(lif, 1.0)
    taus = [k for k in keep if k.numel() == 20 and float(k.max()) == 50.0]
    assert taus and torch.equal(taus[0].reshape(4, 5), torch.tensor([10.0, 20.0, 30.0, 40.0, 50.0]).expand(4, 5))
    for bad in (torch.full((2, 8), 20.0), torch.full((3, 1), 20.0)):
        with pytest.raises(NotImplementedError, match="per-sample"):
            _build_neuron_desc(LIF(8, tau=bad), 1.0)


def test_engine_refuses_states_of_different_batch():
    from btorch_b200.models import engine

    n = 16
    rnn = RecurrentNN(LIF(n, tau_ref=2.0), ExponentialPSC(n, 5.0, SparseConn(sp.coo_array(np.eye(n, dtype=np.float32)))))
    init_net_state(rnn, batch_size=3)
    rnn.synapse.reset(batch_size=5)
    plan, _ = rnn.fused_plan()
    with pytest.raises(RuntimeError, match="disagree on the batch size"):
        engine.run(plan, rnn, torch.zeros(4, 3, n))


def test_neuron_step_refuses_states_of_another_batch():
    from btorch_b200.models._ops import neuron_step

    lif = LIF(8, tau_ref=2.0)
    x, v = torch.zeros(3, 8), torch.zeros(3, 8)
    with pytest.raises(RuntimeError, match="does not match the input"):
        neuron_step(lif, x, v, torch.zeros(5, 8), None, 1.0)
    with pytest.raises(RuntimeError, match="CUDA"):  # matching shapes get as far as the device check
        neuron_step(lif, x, v, torch.zeros(3, 8), None, 1.0)


def test_product_package_never_reaches_the_oracle():
    """The oracle is test infrastructure: no module of the package imports,
    loads or names it, so the product path cannot route through it (tests,
    smoke() and the bench's CPU arms are its only callers)."""
    pkg = ROOT / "btorch_b200"
    offenders = [str(p.relative_to(ROOT)) for p in pkg.rglob("*")
                 if p.suffix in (".py", ".cu", ".cuh", ".cpp", ".h")
                 and re.search(r"\boracle\b|liboracle|orc_run", p.read_text())]
    assert offenders == []
    import subprocess
    import sys

    # a fresh interpreter importing the whole module API loads no oracle module
    code = ("import sys, btorch_b200, btorch_b200.models, btorch_b200.serving, btorch_b200.io, "
            "btorch_b200.connectome; print(any(m == 'oracle' or m.startswith('oracle.') for m in sys.modules))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.strip().splitlines()[-1] == "False"


def test_tile_mode_is_an_opt_in_candidate():
    """The persistent tile engine is a tuner candidate only when the sparse
    config asks for it, for networks without delays or receptor channels, in
    a push direction and batches up to 256."""
    from btorch_b200.models import autotune

    conn = SparseConn(sp.random(64, 64, density=0.1, random_state=0, format="coo", dtype=np.float32),
                      sparse_config={"direction": "scatter"})
    assert L.BT_MODE_TILE not in autotune.allowed_modes(conn, 8)
    conn.sparse_config.tile = True
    assert L.BT_MODE_TILE in autotune.allowed_modes(conn, 8)
    assert L.BT_MODE_TILE not in autotune.allowed_modes(conn, 8, n_bins=3)
    assert L.BT_MODE_TILE not in autotune.allowed_modes(conn, 8, receptors=2)
    assert L.BT_MODE_TILE not in autotune.allowed_modes(conn, 300)
    conn.sparse_config.direction = "gather"
    assert L.BT_MODE_TILE not in autotune.allowed_modes(conn, 8)


def test_cluster_mode_is_a_candidate_unless_scatter_is_asked_for():
    """The single-cluster engine (an ordered gather) is offered with
    direction auto or gather, deterministic included, with up to 32 delay
    bins, but not with an explicit scatter, receptor channels or more than
    256 samples."""
    import scipy.sparse as sp

    from btorch_b200.models import SparseConn, autotune

    conn = SparseConn(sp.coo_array(np.eye(64, dtype=np.float32)), sparse_config={"direction": "auto"})
    assert L.BT_MODE_CLUSTER in autotune.allowed_modes(conn, 8)
    assert L.BT_MODE_CLUSTER not in autotune.allowed_modes(conn, 8, receptors=2)
    assert L.BT_MODE_CLUSTER in autotune.allowed_modes(conn, 8, n_bins=3)
    assert L.BT_MODE_CLUSTER not in autotune.allowed_modes(conn, 8, n_bins=40)
    assert L.BT_MODE_CLUSTER not in autotune.allowed_modes(conn, 300)
    conn.sparse_config.direction = "gather"
    assert L.BT_MODE_CLUSTER in autotune.allowed_modes(conn, 8)
    conn.sparse_config.deterministic = True
    assert L.BT_MODE_CLUSTER in autotune.allowed_modes(conn, 8)
    conn.sparse_config.deterministic = False
    conn.sparse_config.direction = "scatter"
    assert L.BT_MODE_CLUSTER not in autotune.allowed_modes(conn, 8)


@pytest.mark.parametrize("n,tp", [(300, 32), (1000, 128), (4096, 256)])
def test_cluster_packing_holds_every_in_edge_in_order(n, tp):
    """The cluster engine's packed in-edges, read back the way the kernel
    walks them (tile, slice, lane: groups of 4 rows in order), list every
    post's in-edges in ascending canonical order, with id XOR 31 and the
    weight, and only padding (id n, weight 0) after them."""
    from btorch_b200.models import SparseConn
    from btorch_b200.models._ops import pack_slice_weights
    from btorch_b200.models.engine import cluster_pack, cluster_pack_index, cluster_shape, slices_of

    rng = np.random.default_rng(n)
    dense = (rng.random((n, n)) < min(0.03, 80.0 / n)) * rng.normal(0, 1, (n, n))
    conn = SparseConn(sp.coo_array(dense.astype(np.float32)))
    lay = conn.engine_layout(1, 0, "cpu")
    sl = slices_of(lay, "cpu")
    shape = cluster_shape(n, 1, lay.slices_ptr_host, ctas=-(-n // tp))
    assert shape is not None and shape[0] == tp
    tp, P, rows = shape
    index, gptr = cluster_pack_index(lay, n, tp, P, rows, "cpu")
    w = conn._edge_weight().detach().float().contiguous()
    cl_w, cl_src = cluster_pack(sl, pack_slice_weights(sl, w), index, n)
    G = rows // 4
    cw = cl_w.numpy().reshape(P, G, 32, 4)
    cs = cl_src.numpy().astype(np.int64).reshape(P, G, 32, 4) & 0xFFFF if n + 32 <= 65536 else None
    gp = gptr.numpy().reshape(P, tp // 32 + 1)
    csc = dense.T  # [post, pre]
    for t in range(P):
        for s_ in range((min(tp, n - t * tp) + 31) // 32):
            for ln in range(32):
                post = t * tp + s_ * 32 + ln
                got_ids = (cs[t, gp[t, s_]:gp[t, s_ + 1], ln, :].reshape(-1) ^ 31)
                got_w = cw[t, gp[t, s_]:gp[t, s_ + 1], ln, :].reshape(-1)
                if post >= n:
                    assert (got_ids == n).all()
                    continue
                pres = np.nonzero(csc[post])[0]
                k = len(pres)
                np.testing.assert_array_equal(got_ids[:k], pres)
                np.testing.assert_array_equal(got_w[:k], csc[post, pres].astype(np.float32))
                assert (got_ids[k:] == n).all() and (got_w[k:] == 0).all()


def test_cluster_packing_carries_the_delay_bin():
    """With delay bins (here DelayedPSC's uniform delay: every edge in bin 2)
    the packed ids are 32-bit, the id XOR 31 in bits 0..19 and the bin in
    bits 20..24; the padding has bin 0 and id n."""
    from btorch_b200.models import SparseConn
    from btorch_b200.models._ops import pack_slice_weights
    from btorch_b200.models.engine import cluster_pack, cluster_pack_index, cluster_shape, slices_of

    n = 700
    rng = np.random.default_rng(2)
    dense = (rng.random((n, n)) < 0.04) * rng.normal(0, 1, (n, n))
    conn = SparseConn(sp.coo_array(dense.astype(np.float32)))
    lay = conn.engine_layout(3, 2, "cpu")
    sl = slices_of(lay, "cpu")
    tp, P, rows = cluster_shape(n, 2, lay.slices_ptr_host, n_bins=3)
    index, gptr = cluster_pack_index(lay, n, tp, P, rows, "cpu")
    w = conn._edge_weight().detach().float().contiguous()
    cl_w, cl_src = cluster_pack(sl, pack_slice_weights(sl, w), index, n, 3)
    assert cl_src.dtype == torch.int32
    ids = cl_src.numpy().astype(np.int64)
    pre = (ids & 0xFFFFF) ^ 31
    edge = pre != n  # the slices' own padding and the rows added per slice hold id n, bin 0
    assert ((ids[edge] >> 20) == 2).all() and ((ids[~edge] >> 20) == 0).all()
    pres = pre[edge]
    assert pres.max() < n and np.bincount(pres, minlength=n).sum() == int((dense != 0).sum())
    assert L.lib().bt_cluster_smem_bytes(n, 2, tp, rows, 3) > L.lib().bt_cluster_smem_bytes(n, 2, tp, rows, 1)
    assert L.lib().bt_cluster_smem_bytes(n, 2, tp, rows, 33) == 0
