"""Time the reference's own CPU step beside the C port (build-container recipe).

The reference checkout is imported read-only from the directory given by
--ref, or else by the BTORCH_REFERENCE environment variable (it does not
exist where the GPU runs, so the bench cannot do this there).  On the
plain workload (LIF + ExponentialPSC + SparseConn with the reference's
native sparse backend, DenseConn input, N 4096, p 0.02, batch 1) it runs
the reference's RecurrentNN for --steps steps and the port (oracle/oracle.c,
the CPU baseline the bench reports) for the same steps on the same inputs,
each with --threads host threads, and prints one JSON line: milliseconds
per step of each, their ratio, and whether the two spike rasters agree.

    BTORCH_REFERENCE=<reference checkout> python oracle/time_reference_cpu.py --steps 200
"""

from __future__ import annotations

import argparse
import importlib.metadata as md
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("BTORCH_REFERENCE"))
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or BTORCH_REFERENCE")
    orig = md.version
    md.version = lambda name: "0.0.0+ref" if name == "btorch" else orig(name)
    sys.path.insert(0, args.ref)
    sys.path.insert(0, str(ROOT))
    import scipy.sparse as sp
    import torch

    import bench
    from btorch.models import environ
    from btorch.models.functional import init_net_state
    from btorch.models.linear import DenseConn, SparseConn
    from btorch.models.neurons import LIF
    from btorch.models.rnn import RecurrentNN
    from btorch.models.synapse import ExponentialPSC
    from oracle import oracle as O

    torch.set_num_threads(args.threads)
    cfg = dict(bench.CONFIGS["plain"])
    n, T = cfg["n"], args.steps
    net = bench.make_network(cfg, 0)
    x, _ = bench.host_inputs(cfg, 0, T)
    x = np.ascontiguousarray(np.asarray(x)[:T], dtype=np.float32)

    # the reference's own modules (its native sparse backend on the CPU)
    w_pre_post = sp.coo_array((net["w"], (net["src"], net["post"])), shape=(n, n))
    conn = SparseConn(w_pre_post, sparse_backend="native")
    neuron = LIF(n, v_threshold=1.0, v_reset=0.0, tau=20.0, tau_ref=2.0, hard_reset=True)
    syn = ExponentialPSC(n, tau_syn=5.0, linear=conn)
    inp = DenseConn(cfg["c_in"], n, weight=torch.from_numpy(net["w_in"]))
    brain = RecurrentNN(neuron, syn, neuron_inp_module=inp, update_state_names=())
    init_net_state(brain, batch_size=1, dtype=torch.float32)
    with torch.no_grad(), environ.context(dt=1.0):
        t0 = time.perf_counter()
        z_ref, _ = brain(torch.from_numpy(x))
        ref_s = time.perf_counter() - t0
    z_ref = z_ref.numpy().astype(np.uint8)

    # the port, as the bench's CPU baseline runs it
    t0 = time.perf_counter()
    _, _, threads, z_port = bench.cpu_sample(cfg, net, x, T)
    port_s = time.perf_counter() - t0
    same = int(np.array_equal(np.asarray(z_port).astype(np.uint8).reshape(z_ref.shape), z_ref))
    print(json.dumps({"workload": bench.describe("plain", cfg), "steps": T, "threads": args.threads,
                      "reference_ms_per_step": 1e3 * ref_s / T, "port_ms_per_step": 1e3 * port_s / T,
                      "reference_over_port": ref_s / port_s, "rasters_equal": bool(same),
                      "port_threads": threads}))


if __name__ == "__main__":
    main()
