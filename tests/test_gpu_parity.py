"""GPU parity: the sm_100a kernels against the reference's golden vectors and
the CPU oracle, through the module API (which calls the C ABI)."""

import operator
import numpy as np
import pytest
import torch

from btorch_b200.models import environ
from oracle import oracle as O
from tests import cases

pytestmark = pytest.mark.gpu
DEV = "cuda"


def first_divergence(a, b):
    bad = np.nonzero((a != b).reshape(len(a), -1).any(1))[0]
    return int(bad[0]) if bad.size else len(a)


def run_engine(d, direction, chunk=None, names_out=False):
    rnn, psc_name = cases.build_model(d, DEV, direction)
    with torch.no_grad(), environ.context(dt=float(d["dt"])):
        z, st = rnn(torch.tensor(d["x"], device=DEV), engine_chunk=chunk)
    assert rnn.last_path == "fused"
    out = {"z": z.cpu().numpy().astype(np.uint8), "v": st["neuron.v"].cpu().numpy(),
           "psc": st[psc_name].cpu().numpy(), "v_final": rnn.neuron.v.cpu().numpy(), "rnn": rnn}
    return out


# ----------------------------------------------------------------- sparse op --

def _spmm_module(d, direction):
    import scipy.sparse as sp

    from btorch_b200.models import SparseConn

    W = sp.coo_array((d["w"], (d["src"], d["post"])), shape=(int(d["n_in"]), int(d["n_out"])))
    return SparseConn(W, enforce_dale=False, sparse_config={"direction": direction}).to(DEV)


def test_spmv_gather_is_bitwise_reference():
    d = cases.load("spmm_graded")
    m = _spmm_module(d, "gather")
    with torch.no_grad():
        out = m(torch.tensor(d["x"], device=DEV)).cpu().numpy()
    np.testing.assert_array_equal(out, d["out"])


def test_spmv_scatter_matches_reference():
    d = cases.load("spmm_graded")
    m = _spmm_module(d, "scatter")
    with torch.no_grad():
        out = m(torch.tensor(d["x"], device=DEV)).cpu().numpy()
    np.testing.assert_allclose(out, d["out"], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("direction", ["gather", "scatter"])
def test_spmv_backward_matches_reference_autograd(direction):
    d = cases.load("spmm_graded")
    m = _spmm_module(d, direction)
    x = torch.tensor(d["x"], device=DEV, requires_grad=True)
    out = m(x)
    (out * torch.tensor(d["g"], device=DEV)).sum().backward()
    np.testing.assert_allclose(x.grad.cpu().numpy(), d["grad_x"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(m.magnitude.grad.cpu().numpy(), d["grad_w"], rtol=1e-5, atol=1e-5)


def test_spmv_one_dim_and_leading_dims():
    d = cases.load("spmm_graded")
    m = _spmm_module(d, "gather")
    x = torch.tensor(d["x"], device=DEV)
    with torch.no_grad():
        full = m(x)
        one = m(x[0])
        lead = m(x.reshape(1, *x.shape))
    assert one.shape == (int(d["n_out"]),)
    torch.testing.assert_close(one, full[0], rtol=0, atol=0)
    torch.testing.assert_close(lead[0], full, rtol=0, atol=0)


def test_spmv_gather_deterministic_and_empty_input():
    d = cases.load("spmm_graded")
    m = _spmm_module(d, "gather")
    x = torch.tensor(d["x"], device=DEV)
    with torch.no_grad():
        a, b = m(x), m(x)
        z = m(torch.zeros_like(x))
    assert torch.equal(a, b)
    assert float(z.abs().sum()) == 0.0


# ---------------------------------------------------------- fused engine --

BITWISE_LIF = ["lif_dyadic_soft", "lif_dyadic_input", "delayed_psc", "hetero_delay"]


MODES = ["gather", "pull", "scatter"]


@pytest.mark.parametrize("direction", MODES)
@pytest.mark.parametrize("name", BITWISE_LIF)
def test_engine_bitwise_vs_reference_dyadic(name, direction):
    """Dyadic weights: spike rasters, traces and final state bit-identical to
    the reference's own CPU run, in both directions."""
    d = cases.load(name)
    out = run_engine(d, direction)
    ref_z = cases.spikes(d)
    K = d["v"].shape[0]
    assert first_divergence(out["z"], ref_z) == len(ref_z)
    np.testing.assert_array_equal(out["v"][:K].reshape(d["v"].shape), d["v"])
    np.testing.assert_array_equal(out["psc"][:K].reshape(d["psc"].shape), d["psc"])
    np.testing.assert_array_equal(out["v_final"].reshape(d["v_final"].shape), d["v_final"])


@pytest.mark.parametrize("direction", ["gather", "pull"])
def test_engine_gather_bitwise_vs_reference_nondyadic_recurrence(direction):
    """Non-dyadic lognormal weights (C1-shaped): the ordered gather reproduces
    the reference's fmaf order, so with the same projected input the whole
    run is bit-identical.  The projected input comes from the oracle's ordered
    projection, which the CUDA projection matches bit for bit."""
    d = cases.load("lif_c1_small")
    out = run_engine(d, direction)
    spec = cases.netspec(d)
    st = O.init_state(spec, int(d["batch"]))
    o = O.run(spec, st, cases.projected_input(d, use_reference_projection=False), want_v=True, want_psc=True)
    assert first_divergence(out["z"], o["spikes"]) == len(o["spikes"])
    np.testing.assert_array_equal(out["v"], o["v"])
    np.testing.assert_array_equal(out["psc"], o["psc"])


def test_engine_input_projection_close_to_reference_mkl():
    """Against the reference itself (MKL-ordered projection): traces agree
    within rel 1e-5 until the first spike divergence."""
    d = cases.load("lif_c1_small")
    out = run_engine(d, "gather")
    ref_z = cases.spikes(d)
    k = first_divergence(out["z"], ref_z)
    K = min(k, d["v"].shape[0])
    assert K >= 5
    np.testing.assert_allclose(out["v"][:K], d["v"][:K], rtol=1e-5, atol=1e-5)


def test_engine_scatter_nondyadic_close():
    d = cases.load("lif_c1_small")
    g = run_engine(d, "gather")
    s = run_engine(d, "scatter")
    k = first_divergence(g["z"], s["z"])
    assert k >= 20
    np.testing.assert_allclose(s["v"][:k], g["v"][:k], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("direction", MODES)
def test_engine_alif_vs_reference(direction):
    d = cases.load("alif_exppsc")
    out = run_engine(d, direction)
    ref_z = cases.spikes(d)
    K = d["v"].shape[0]
    k = first_divergence(out["z"], ref_z)
    assert k >= K, f"spikes diverged at {k}"
    np.testing.assert_allclose(out["v"][:K], d["v"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(out["psc"][:K], d["psc"], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("name", ["delayed_psc", "hetero_delay", "lif_dyadic_input"])
@pytest.mark.parametrize("direction", MODES)
def test_engine_split_calls_equal_one_call(name, direction):
    """Two consecutive calls (state, delay history and pending currents carried
    in the modules) equal one call; chunked launches equal one chunk."""
    d = cases.load(name)
    full = run_engine(d, direction)
    rnn, psc_name = cases.build_model(d, DEV, direction)
    x = torch.tensor(d["x"], device=DEV)
    T1 = 37
    with torch.no_grad(), environ.context(dt=float(d["dt"])):
        z1, _ = rnn(x[:T1])
        z2, _ = rnn(x[T1:], engine_chunk=16)
    z = torch.cat([z1, z2]).cpu().numpy().astype(np.uint8)
    np.testing.assert_array_equal(z, full["z"])
    np.testing.assert_array_equal(rnn.neuron.v.cpu().numpy(), full["v_final"])


@pytest.mark.parametrize("direction", MODES)
def test_engine_uneven_sample_lengths(direction):
    """A batch with per-sample lengths equals each sample run alone for its length."""
    d = cases.load("lif_dyadic_soft")
    lens = [120, 47, 1, 90]
    rnn, _ = cases.build_model(d, DEV, direction)
    x = torch.tensor(d["x"], device=DEV)
    with torch.no_grad(), environ.context(dt=1.0):
        z, st = rnn(x, sample_len=torch.tensor(lens))
    z = z.cpu().numpy()
    v_final = rnn.neuron.v.cpu().numpy()
    ref_z = cases.spikes(d)
    spec = cases.netspec(d)
    for b, L in enumerate(lens):
        np.testing.assert_array_equal(z[:L, b], ref_z[:L, b])
        assert z[L:, b].sum() == 0
        stb = O.init_state(spec, 1)
        O.run(spec, stb, d["x"][:L, b: b + 1])
        np.testing.assert_array_equal(v_final[b], stb.v[0])


@pytest.mark.parametrize("direction", ["gather", "pull"])
def test_modular_path_equals_fused_engine(direction):
    """Stepping module by module (each module's own kernel) gives the same run."""
    d = cases.load("hetero_delay")
    fused = run_engine(d, direction)
    assert fused["rnn"].last_engine_direction == direction
    rnn, psc_name = cases.build_model(d, DEV, "gather")
    rnn.fused = False
    with torch.no_grad(), environ.context(dt=1.0):
        z, st = rnn(torch.tensor(d["x"], device=DEV))
    assert rnn.last_path == "modular"
    np.testing.assert_array_equal(z.cpu().numpy().astype(np.uint8), fused["z"])
    np.testing.assert_array_equal(st["neuron.v"].cpu().numpy(), fused["v"])


@pytest.mark.parametrize("direction", MODES)
def test_engine_state_names_default_all_memories(direction):
    """update_state_names=None returns every memory stacked over time, like the
    reference (including the delay history)."""
    d = cases.load("delayed_psc")
    rnn, _ = cases.build_model(d, DEV, direction)
    rnn.update_state_names = None
    rnn_m, _ = cases.build_model(d, DEV, "gather")
    rnn_m.update_state_names = None
    rnn_m.fused = False
    x = torch.tensor(d["x"][:30], device=DEV)
    with torch.no_grad(), environ.context(dt=1.0):
        _, st_f = rnn(x)
        _, st_m = rnn_m(x)
    assert rnn.last_path == "fused" and rnn_m.last_path == "modular"
    assert sorted(st_f) == sorted(st_m)
    for k in st_f:
        torch.testing.assert_close(st_f[k], st_m[k], rtol=0, atol=0, msg=k)


@pytest.mark.parametrize("direction", MODES)
@pytest.mark.parametrize("name", ["lif_dyadic_input", "hetero_delay"])
def test_uneven_lengths_without_traces(name, direction):
    """Per-sample lengths with no state traces requested (finished samples are
    then neither read nor written, and their projected input rows are not
    computed): every sample's raster and final state (v, psc) equal the same
    sample run alone for its length, and spikes after its end are zero."""
    d = cases.load(name)
    B = int(d["batch"])
    T = d["x"].shape[0]
    lens = [T, 31, 1, 77][:B]
    rnn, psc_name = cases.build_model(d, DEV, direction)
    rnn.update_state_names = ()
    x = torch.tensor(d["x"], device=DEV)
    with torch.no_grad(), environ.context(dt=float(d["dt"])):
        z, _ = rnn(x, sample_len=torch.tensor(lens))
    z = z.cpu().numpy()
    v = rnn.neuron.v.cpu().numpy()
    psc = operator.attrgetter(psc_name)(rnn).cpu().numpy()
    for b, L in enumerate(lens):
        alone, _ = cases.build_model(dict(d, batch=np.int64(1)), DEV, direction)
        alone.update_state_names = ()
        with torch.no_grad(), environ.context(dt=float(d["dt"])):
            za, _ = alone(x[:L, b:b + 1])
        np.testing.assert_array_equal(z[:L, b], za.cpu().numpy()[:, 0], err_msg=f"sample {b}")
        assert z[L:, b].sum() == 0
        np.testing.assert_array_equal(v[b], alone.neuron.v.cpu().numpy()[0])
        np.testing.assert_array_equal(psc[b], operator.attrgetter(psc_name)(alone).cpu().numpy()[0])


@pytest.mark.parametrize("batch", [1, 37, 128, 200])
def test_grad_input_transposed_matches_lane_split(batch):
    """bt_spmv_grad_input_t (gradient transposed into scratch, one contiguous
    sample run per edge) against bt_spmv_grad_input and a float64 product:
    both fp32 sums within 1e-5, the transposed one deterministic."""
    import scipy.sparse as sp

    from btorch_b200 import _lib as L
    from btorch_b200.models import SparseConn
    from btorch_b200.models._ops import pack_csr_weights

    rng = np.random.default_rng(batch)
    n_in, n_out = 700, 900
    W = sp.random(n_in, n_out, density=0.03, random_state=batch, dtype=np.float32)
    m = SparseConn(sp.coo_array(W), enforce_dale=False).to(DEV)
    lay = m.layout(DEV)
    w_csr = pack_csr_weights(lay, m._get_effective_weight().detach())
    g = torch.tensor(rng.standard_normal((batch, n_out)).astype(np.float32), device=DEV)
    outs = []
    s = L.stream_of(torch.device(DEV))
    for fn in ("bt_spmv_grad_input", "bt_spmv_grad_input_t", "bt_spmv_grad_input_t"):
        gx = torch.empty((batch, n_in), device=DEV)
        args = [batch, n_in, n_out, lay.csr_ptr.data_ptr(), lay.csr_dst.data_ptr(), w_csr.data_ptr(), g.data_ptr(),
                gx.data_ptr()]
        if fn.endswith("_t"):
            work = torch.empty(batch * n_out, device=DEV)
            args.append(work.data_ptr())
        L.check(getattr(L.lib(), fn)(*args, s), fn)
        outs.append(gx.cpu().numpy())
    want = g.cpu().numpy().astype(np.float64) @ W.toarray().astype(np.float64).T
    np.testing.assert_allclose(outs[0], want, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(outs[1], want, rtol=1e-5, atol=1e-5)
    np.testing.assert_array_equal(outs[1], outs[2])


def test_input_project_live_rows_equal_full_projection():
    """bt_input_project_live writes exactly the rows of live steps, equal to
    bt_input_project's, and leaves the rows of finished samples untouched."""
    from btorch_b200 import _lib as L

    rng = np.random.default_rng(3)
    steps, batch, c_in, n = 9, 5, 300, 1100
    x = torch.tensor((rng.random((steps, batch, c_in)) < 0.05).astype(np.float32) * 1.5, device=DEV)
    w_t = torch.tensor(rng.standard_normal((c_in, n)).astype(np.float32), device=DEV)
    bias = torch.tensor(rng.standard_normal(n).astype(np.float32), device=DEV)
    lens = torch.tensor([9, 0, 4, 1, 7], dtype=torch.int32, device=DEV)
    work = torch.empty(steps * batch * (2 * c_in + 1), dtype=torch.int32, device=DEV)
    s = L.stream_of(torch.device(DEV))
    full = torch.empty((steps, batch, n), device=DEV)
    L.check(L.lib().bt_input_project(steps * batch, c_in, n, x.data_ptr(), w_t.data_ptr(), bias.data_ptr(),
                                     full.data_ptr(), work.data_ptr(), s), "bt_input_project")
    live = torch.full((steps, batch, n), 1234.5, device=DEV)
    L.check(L.lib().bt_input_project_live(steps, batch, c_in, n, x.data_ptr(), w_t.data_ptr(), bias.data_ptr(),
                                          lens.data_ptr(), live.data_ptr(), work.data_ptr(), s),
            "bt_input_project_live")
    f, lv = full.cpu().numpy(), live.cpu().numpy()
    for b, L_b in enumerate(lens.tolist()):
        np.testing.assert_array_equal(lv[:L_b, b], f[:L_b, b])
        assert (lv[L_b:, b] == 1234.5).all()
