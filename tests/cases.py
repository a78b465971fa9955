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
