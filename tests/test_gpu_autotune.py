"""The engine autotuner: it times the candidates allowed by the sparse config on
the caller's model, caches the winner, restores the state after its trials,
and the tuned run equals the untuned one bit for bit (dyadic weights)."""

import numpy as np
import pytest
import torch

from btorch_b200.models import autotune, environ
from tests import cases

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _conn(rnn):
    syn = rnn.synapse
    for m in (syn, getattr(syn, "psc_module", None), getattr(syn, "base_psc", None)):
        if m is not None and hasattr(m, "linear"):
            return m.linear
    raise AssertionError("no SparseConn")


@pytest.mark.parametrize("direction", ["scatter", "gather", "auto"])
@pytest.mark.parametrize("name", ["hetero_delay", "lif_dyadic_input"])
def test_tuned_run_equals_untuned(name, direction):
    d = cases.load(name)
    T = autotune.TUNE_MIN_STEPS + 44
    x = torch.tensor(np.concatenate([d["x"]] * (T // len(d["x"]) + 1))[:T], device=DEV)
    outs = {}
    for tune in (False, True):
        rnn, _ = cases.build_model(d, DEV, "scatter")
        conn = _conn(rnn)
        conn.sparse_config.direction = direction
        conn.sparse_config.autotune = tune
        with torch.no_grad(), environ.context(dt=float(d["dt"])):
            z, st = rnn(x)
            z2, _ = rnn(x[:50])
        outs[tune] = (z.cpu().numpy(), st["neuron.v"].cpu().numpy(), z2.cpu().numpy(), rnn.neuron.v.cpu().numpy())
        if tune:
            cache = autotune.tuned(rnn)
            assert len(cache) == 1
            best, timings = next(iter(cache.values()))
            n_bins = int(d["n_bins"]) if int(d["n_bins"]) > 1 else 1
            cands = autotune.candidates(conn, int(d["batch"]), 1, n_bins, int(d["n"]), rnn.neuron.v.device)
            assert set(timings) == set(cands) and best in cands
            assert rnn.last_engine_choice == best
            assert best.mode in autotune.allowed_modes(conn, int(d["batch"]), 1, n_bins)
    for a, b in zip(outs[False], outs[True]):
        np.testing.assert_array_equal(a, b)


def test_explicit_engine_choice_is_used():
    """engine_choice= bypasses the tuner: the run uses it and equals the tuned run."""
    from btorch_b200 import _lib as L

    d = cases.load("lif_dyadic_input")
    x = torch.tensor(d["x"], device=DEV)
    outs = []
    for choice in (None, autotune.EngineChoice(L.BT_MODE_SCATTER, neuron_spt=1, scatter_lanes=8)):
        rnn, _ = cases.build_model(d, DEV, "scatter")
        with torch.no_grad(), environ.context(dt=float(d["dt"])):
            z, _ = rnn(x, engine_choice=choice)
        if choice is not None:
            assert rnn.last_engine_choice == choice
        outs.append(z.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
