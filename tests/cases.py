"""Golden cases (made from the reference by tests/golden/make_golden.py) as
oracle NetSpecs and module-level configurations."""

from __future__ import annotations

from pathlib import Path

import numpy as np

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
STEP_CASES = ["lif_c1_small", "lif_dyadic_soft", "lif_dyadic_input", "alif_exppsc", "delayed_psc", "hetero_delay"]


def load(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as f:
        return {k: f[k] for k in f.files}


def spikes(d: dict) -> np.ndarray:
    """Unpacked reference raster [T, B, n] (uint8)."""
    return np.unpackbits(d["z"], axis=-1, bitorder="little")[..., : int(d["n"])]


def csc(d: dict):
    """Canonical CSC arrays (ptr, pre, delay, w) from the golden COO."""
    n = int(d["n"])
    n_bins = int(d["n_bins"])
    post, src, w = d["post"], d["src"], d["w"]
    ptr = np.zeros(n + 1, np.int64)
    np.add.at(ptr, post + 1, 1)
    ptr = np.cumsum(ptr)
    pre = (src // n_bins).astype(np.int32)
    delay = (src % n_bins).astype(np.int32) + int(d["uniform_delay"])
    return ptr, pre, delay, w.astype(np.float32)


def netspec(d: dict) -> O.NetSpec:
    ptr, pre, delay, w = csc(d)
    kind = int(d["kind"])
    P = {"v_threshold": d["vth"], "v_reset": d["vr"], "c_m": d["cm"], "psc_coef": d["psc_coef"],
         "psc_tau": d["psc_tau"]}
    if kind == 0:
        P["tau"] = d["tau"]
    else:
        for k in ("g_leak", "E_leak", "E_k", "dg_k", "tau_adapt", "coef_gk"):
            P[k] = d[k]
    if int(d["use_ref"]):
        P["tau_ref"] = d["tau_ref"]
    return O.NetSpec(n=int(d["n"]), kind=kind, hard_reset=bool(d["hard"]), use_ref=bool(d["use_ref"]),
                     dt=float(d["dt"]), params=P, ptr=ptr, pre=pre, delay=delay, w=w,
                     max_delay=int(delay.max()) if delay.size else 0)


def projected_input(d: dict, use_reference_projection: bool = True) -> np.ndarray:
    """The per-neuron input current [T, B, n]: x itself, or the DenseConn
    projection (the reference's own MKL result, or the oracle's ordered one)."""
    x = d["x"]
    if "W_in" not in d:
        return x
    if use_reference_projection:
        return d["x_proj_ref"]
    T, B, c = x.shape
    return O.linear(x.reshape(T * B, c), d["W_in"].T).reshape(T, B, -1)


def build_model(d: dict, device="cuda", direction="gather"):
    """The golden case's network built from btorch_b200 modules."""
    import pandas as pd
    import scipy.sparse as sp
    import torch

    from btorch_b200.models import ALIF, LIF, DelayedPSC, DenseConn, ExponentialPSC, HeterSynapsePSC, RecurrentNN
    from btorch_b200.models import SparseConn
    from btorch_b200.models.functional import init_net_state

    n = int(d["n"])
    n_bins = int(d["n_bins"])
    conn_m = sp.coo_array((d["w"], (d["src"], d["post"])), shape=(n * n_bins, n))
    # "gather": ordered pull, warp per post; "pull": ordered pull, sliced lane per post
    cfg = {"gather": {"direction": "gather", "pull_min_batch": 1 << 30},
           "pull": {"direction": "gather", "pull_min_batch": 1},
           "scatter": {"direction": "scatter"}}[direction]
    conn = SparseConn(conn_m, sparse_config=cfg)
    tau_ref = float(d["tau_ref"]) if int(d["use_ref"]) else None
    if int(d["kind"]) == 0:
        neuron = LIF(n, v_threshold=float(d["vth"]), v_reset=float(d["vr"]), c_m=float(d["cm"]),
                     tau=float(d["tau"]), tau_ref=tau_ref, hard_reset=bool(d["hard"]))
    else:
        neuron = ALIF(n, v_threshold=float(d["vth"]), v_reset=float(d["vr"]), c_m=float(d["cm"]),
                      g_leak=float(d["g_leak"]), E_leak=float(d["E_leak"]), E_k=float(d["E_k"]),
                      tau_adapt=float(d["tau_adapt"]), dg_k=float(d["dg_k"]), tau_ref=tau_ref,
                      hard_reset=bool(d["hard"]))
    tau_syn = float(d["psc_tau"])
    D = int(d["uniform_delay"])
    if n_bins > 1:
        rti = pd.DataFrame({"receptor_type": ["syn"], "receptor_index": [0]})
        syn = HeterSynapsePSC(n, 1, rti, conn, base_psc=ExponentialPSC, max_delay_steps=n_bins,
                              use_circular_buffer=True, tau_syn=tau_syn)
        psc_name = "synapse.psc"
    elif D:
        syn = DelayedPSC(ExponentialPSC(n, tau_syn, conn), max_delay_steps=D, use_circular_buffer=True)
        psc_name = "synapse.psc_module.psc"
    else:
        syn = ExponentialPSC(n, tau_syn, conn)
        psc_name = "synapse.psc"
    inp = None
    if "W_in" in d:
        inp = DenseConn(d["W_in"].shape[0], n, weight=torch.tensor(d["W_in"]))
    names = ["neuron.v", psc_name] + (["neuron.g_k"] if int(d["kind"]) == 1 else [])
    rnn = RecurrentNN(neuron, syn, neuron_inp_module=inp, update_state_names=names).to(device)
    init_net_state(rnn, batch_size=int(d["batch"]), dtype=torch.float32, device=device)
    return rnn, psc_name
