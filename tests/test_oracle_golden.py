"""Pin the CPU oracle to the reference: replay every golden case (made by
running the reference's own modules) through oracle.c."""

import numpy as np
import pytest

from oracle import oracle as O
from tests import cases


@pytest.mark.parametrize("events", [False, True], ids=["dense", "events"])
@pytest.mark.parametrize("name", cases.STEP_CASES)
def test_oracle_reproduces_reference_rasters(name, events, cpu_threads):
    """Both synapse phases (every synapse, as the reference computes it; and
    the event-driven push used for full-size parity) against the reference."""
    d = cases.load(name)
    spec = cases.netspec(d)
    st = O.init_state(spec, int(d["batch"]))
    out = O.run(spec, st, cases.projected_input(d), threads=cpu_threads, want_v=True, want_psc=True,
                events=events)
    ref_z = cases.spikes(d)
    K = d["v"].shape[0]
    if int(d["kind"]) == 0:
        # LIF: every op is the reference's op -> bit-identical everywhere
        np.testing.assert_array_equal(out["spikes"], ref_z)
        np.testing.assert_array_equal(out["v"][:K], d["v"])
        np.testing.assert_array_equal(out["psc"][:K], d["psc"])
        np.testing.assert_array_equal(st.v, d["v_final"])
        np.testing.assert_array_equal(st.psc, d["psc_final"])
    else:
        # ALIF: expm1 of the state-dependent term comes from a different libm
        # (last-ulp differences): traces within rel 1e-5 until spikes diverge
        div = np.nonzero((out["spikes"] != ref_z).reshape(len(ref_z), -1).any(1))[0]
        first = int(div[0]) if div.size else len(ref_z)
        assert first >= K, f"spike raster diverged at step {first}"
        np.testing.assert_allclose(out["v"][:K], d["v"], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(out["psc"][:K], d["psc"], rtol=1e-5, atol=1e-6)


def test_oracle_spmm_matches_reference_bitwise():
    d = cases.load("spmm_graded")
    n_out = int(d["n_out"])
    ptr = np.zeros(n_out + 1, np.int64)
    np.add.at(ptr, d["post"] + 1, 1)
    ptr = np.cumsum(ptr)
    out = O.spmm(ptr, d["src"], d["w"], d["x"], n_out)
    np.testing.assert_array_equal(out, d["out"])


def test_oracle_linear_close_to_reference_mkl():
    d = cases.load("lif_c1_small")
    x = d["x"]
    T, B, c = x.shape
    ours = O.linear(x.reshape(T * B, c), d["W_in"].T).reshape(T, B, -1)
    np.testing.assert_allclose(ours, d["x_proj_ref"], rtol=1e-5, atol=1e-6)


def test_oracle_reproduces_training_forward_raster():
    """The training fixture's forward (two truncated-BPTT windows, state
    carried between them) equals the oracle's run over the whole input."""
    import torch

    d = cases.load("train_spiking")
    n, B = int(d["n"]), int(d["batch"])
    ptr = np.zeros(n + 1, np.int64)
    np.add.at(ptr, d["post"] + 1, 1)
    lin = -1.0 / torch.as_tensor(float(d["psc_tau"]))
    coef = float(torch.expm1(lin) / lin)
    spec = O.NetSpec(n=n, kind=0, hard_reset=True, use_ref=True, dt=1.0,
                     params={"v_threshold": 1.0, "v_reset": 0.0, "c_m": 1.0, "tau": float(d["tau"]),
                             "tau_ref": float(d["tau_ref"]), "psc_coef": coef, "psc_tau": float(d["psc_tau"])},
                     ptr=np.cumsum(ptr), pre=d["src"].astype(np.int32), delay=np.zeros(len(d["src"]), np.int32),
                     w=d["w"])
    x = d["x"]
    T = x.shape[0]
    xp = O.linear(x.reshape(T * B, -1), d["W_in"].T.copy()).reshape(T, B, n)
    z = O.run(spec, O.init_state(spec, B), xp)["spikes"]
    np.testing.assert_array_equal(z, np.unpackbits(d["z"], axis=-1, bitorder="little")[..., :n])


@pytest.mark.parametrize("name", ["receptors2", "receptors_delay"])
def test_oracle_receptor_channels_match_reference(name):
    """The oracle's receptor columns (C PSCs per neuron, per-column time
    constants, receptor sum in torch's CPU order) against the reference's
    HeterSynapsePSC runs: rasters, v, per-channel psc and final state bit for
    bit."""
    import torch

    d = cases.load(name)
    n, B, C = int(d["n"]), int(d["batch"]), int(d["n_rec"])
    D = int(d["n_bins"]) if "n_bins" in d else 1
    post, src, w = d["post"].astype(np.int64), d["src"].astype(np.int64), d["w"].astype(np.float32)
    ptr = np.concatenate([[0], np.cumsum(np.bincount(post, minlength=n * C))]).astype(np.int64)
    taus = np.tile(d["taus"].astype(np.float32), n)
    lin = -1.0 / torch.tensor(taus)
    coef = (torch.expm1(1.0 * lin) / lin).numpy()
    spec = O.NetSpec(n=n, kind=0, hard_reset=True, use_ref=True, dt=1.0,
                     params={"v_threshold": 1.0, "v_reset": 0.0, "c_m": 1.0, "tau": 20.0, "tau_ref": 2.0,
                             "psc_coef": coef, "psc_tau": taus},
                     ptr=ptr, pre=(src // D).astype(np.int32), delay=(src % D).astype(np.int32), w=w,
                     max_delay=D - 1, n_rec=C)
    st = O.init_state(spec, B)
    o = O.run(spec, st, d["x"], want_v=True, want_psc=True, threads=4)
    np.testing.assert_array_equal(o["spikes"], cases.spikes(d))
    K = d["v"].shape[0]
    np.testing.assert_array_equal(o["v"][:K], d["v"])
    np.testing.assert_array_equal(o["psc"][:K], d["psc_rec"])
    np.testing.assert_array_equal(st.v, d["v_final"])
    np.testing.assert_array_equal(st.psc, d["psc_rec_final"])


@pytest.mark.parametrize("n_rec", [1, 3])
@pytest.mark.parametrize("kind", [0, 1])
def test_oracle_event_push_equals_synapse_chain(kind, n_rec, cpu_threads):
    """The event-driven synapse phase is bit-identical to the full fmaf chain
    on non-dyadic weights (the order of every column's terms is kept), with
    per-synapse delays, receptor columns, uneven sample lengths and a state
    carried across two calls."""
    rng = np.random.default_rng(11 + kind + 7 * n_rec)
    n, B, T, D = 150, 5, 90, 4
    nc = n * n_rec
    post = np.repeat(np.arange(nc), rng.integers(0, 25, nc))
    pre = rng.integers(0, n, post.size)
    delay = rng.integers(0, D, post.size)
    key = np.unique(post * (n * D) + pre * D + delay)
    post, src = key // (n * D), key % (n * D)
    pre, delay = (src // D).astype(np.int32), (src % D).astype(np.int32)
    w = (rng.lognormal(-1.0, 1.0, post.size) * np.where(pre < 120, 0.05, -0.2)).astype(np.float32)
    ptr = np.concatenate([[0], np.cumsum(np.bincount(post, minlength=nc))]).astype(np.int64)
    P = {"v_threshold": 1.0, "v_reset": 0.0, "c_m": 1.0, "tau_ref": 2.0, "psc_coef": 0.8, "psc_tau": 5.0}
    if kind == 0:
        P["tau"] = 20.0
    else:
        P.update(g_leak=0.05, E_leak=0.0, E_k=-1.0, dg_k=0.07, tau_adapt=200.0, coef_gk=0.99)
    spec = O.NetSpec(n=n, kind=kind, hard_reset=True, use_ref=True, dt=1.0, params=P, ptr=ptr, pre=pre,
                     delay=delay, w=w, max_delay=D - 1, n_rec=n_rec)
    x = (rng.poisson(0.15, (T, B, n)) * 0.7).astype(np.float32)
    lens = rng.integers(T // 3, 2 * T, B).astype(np.int32)
    outs = []
    for events in (False, True):
        st = O.init_state(spec, B)
        a = O.run(spec, st, x[:40], sample_len=np.minimum(lens, 40), threads=cpu_threads, want_v=True,
                  want_psc=True, events=events)
        b = O.run(spec, st, x[40:], sample_len=np.clip(lens - 40, 0, None), threads=cpu_threads, want_v=True,
                  want_psc=True, events=events)
        outs.append((a, b, st))
    (a0, b0, s0), (a1, b1, s1) = outs
    assert a0["spikes"].sum() > 100
    for u, v in ((a0, a1), (b0, b1)):
        for key in ("spikes", "v", "psc"):
            np.testing.assert_array_equal(u[key], v[key])
    for key in ("v", "psc", "ref", "gk", "hist"):
        if getattr(s0, key) is not None:
            np.testing.assert_array_equal(getattr(s0, key), getattr(s1, key))


def test_oracle_projection_threads_do_not_change_the_result():
    d = cases.load("lif_c1_small")
    x = d["x"]
    T, B, c = x.shape
    one = O.linear(x.reshape(T * B, c), d["W_in"].T)
    many = O.linear(x.reshape(T * B, c), d["W_in"].T, threads=7)
    np.testing.assert_array_equal(one, many)
    tr = O.linear_t(x.reshape(T * B, c), d["W_in"], threads=3)  # W_in is [c_in, n]
    np.testing.assert_array_equal(one, tr)
