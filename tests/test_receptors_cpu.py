"""Receptor-sum order: the order HeterSynapsePSC and the fused engine use to
add a neuron's receptor PSCs is the order of torch's CPU sum over a
contiguous row (the reference's psc.reshape(..., n, C).sum(-1),
btorch/models/synapse.py:744-747), for every channel count up to 39."""

import numpy as np
import pandas as pd
import pytest
import torch

from btorch_b200.models import ExponentialPSC, HeterSynapsePSC, SparseConn
from btorch_b200.models.synapse import receptor_sum_ordered


@pytest.mark.parametrize("C", list(range(1, 40)))
def test_ordered_sum_equals_torch_cpu_sum(C):
    rng = np.random.default_rng(C)
    a = (rng.standard_normal((7, 333, C)) * np.exp(rng.standard_normal((7, 333, C)) * 3)).astype(np.float32)
    t = torch.tensor(a)
    np.testing.assert_array_equal(receptor_sum_ordered(t).numpy(), t.sum(-1).numpy())


def test_get_psc_lookup_and_shape_errors():
    import scipy.sparse as sp

    n, C = 5, 4
    idx = pd.DataFrame([(0, "E", "E"), (1, "E", "I"), (2, "I", "E"), (3, "I", "I")],
                       columns=["receptor_index", "pre_receptor_type", "post_receptor_type"])
    conn = SparseConn(sp.coo_array(np.eye(n, n * C, dtype=np.float32)))
    syn = HeterSynapsePSC(n, C, idx, conn, base_psc=ExponentialPSC, tau_syn=5.0)
    psc = torch.arange(2 * n * C, dtype=torch.float32).reshape(2, n * C)
    np.testing.assert_array_equal(syn.get_psc(("I", "E"), psc=psc).numpy(), psc.view(2, n, C)[..., 2].numpy())
    np.testing.assert_array_equal(syn.get_psc(3, psc=psc).numpy(), psc.view(2, n, C)[..., 3].numpy())
    assert syn.get_psc(None, psc=psc) is psc
    with pytest.raises(ValueError, match="neuron mode"):
        syn.get_psc("E", psc=psc)
    with pytest.raises(ValueError, match="NaN"):
        syn.get_psc(0, psc=torch.full((1, n * C), float("nan")))
    with pytest.raises(RuntimeError, match="shape mismatch"):
        syn._flatten_input(torch.zeros(2, n + 1))
    flat, lead, has = syn._flatten_input(torch.zeros(3, n, C))
    assert has and tuple(lead) == (3,) and flat.shape == (3, n * C)
