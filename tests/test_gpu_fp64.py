"""FP32 membrane error of the CUDA engine against the reference run in FP64
(tests/golden/fp64_c1.npz: the C1 model at reduced size, 200 steps), stated
as max |v_fp32 - v_fp64| over the first 200 steps."""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from btorch_b200.models import LIF, DenseConn, ExponentialPSC, RecurrentNN, SparseConn, environ
from btorch_b200.models.functional import init_net_state
from tests import cases

pytestmark = pytest.mark.gpu
DEV = "cuda"


@pytest.mark.parametrize("direction", ["gather", "scatter"])
def test_fp32_membrane_error_vs_fp64_reference(direction):
    d = cases.load("fp64_c1")
    n, steps = int(d["n"]), int(d["steps"])
    W = sp.coo_array((d["w"], (d["src"].astype(np.int64), d["post"].astype(np.int64))), shape=(n, n))
    conn = SparseConn(W, sparse_config={"direction": direction})
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True)
    rnn = RecurrentNN(neuron, ExponentialPSC(n, tau_syn=5.0, linear=conn),
                      neuron_inp_module=DenseConn(d["W_in"].shape[0], n, weight=torch.tensor(d["W_in"])),
                      update_state_names=("neuron.v",)).to(DEV)
    init_net_state(rnn, batch_size=1, dtype=torch.float32, device=DEV)
    with torch.no_grad(), environ.context(dt=1.0):
        z, st = rnn(torch.tensor(d["x"], device=DEV))
    z = z.cpu().numpy().astype(np.uint8)
    z64 = np.unpackbits(d["z64"], axis=-1, bitorder="little")[..., :n]
    bad = np.nonzero((z != z64).reshape(steps, -1).any(1))[0]
    k = int(bad[0]) if bad.size else steps
    v = st["neuron.v"].cpu().numpy()[:, :, :64].astype(np.float64)
    err = np.abs(v[:k] - d["v64"][:k]).max()
    # the reference's own fp32 run sits at the same distance from fp64
    ref_err = float(d["err_max"][: int(d["first_divergence"])].max())
    print(f"\n{direction}: raster equal to fp64 for {k}/{steps} steps; max |v32 - v64| = {err:.3g} "
          f"(reference fp32: {ref_err:.3g})")
    assert k == steps
    assert err < 4 * max(ref_err, 1e-7)
