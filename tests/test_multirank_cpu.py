"""The replica path of bench.py (one process per GPU, no data-path
collective): every rank simulates its own batch, the job's time is the slowest
rank's and its work the sum -- checked with two gloo ranks on the CPU."""

import os

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        elapsed = 10.0 + 5.0 * rank          # ms, rank 1 is the slowest
        events = 1000 * (rank + 1)
        t, e = bench.job_totals(elapsed, events, torch.device("cpu"))
        out[rank] = (t, e)
    finally:
        dist.destroy_process_group()


def test_two_replicas_aggregate_max_time_and_total_events():
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1] == (15.0, 3000)


def test_replicas_share_the_network():
    """Every rank builds the same network from the shared seed (weights are
    read-only and replicated); only the inputs are seeded per rank."""
    import bench

    cfg = dict(bench.CONFIGS["batched"], n=64, indeg=8, c_in=16, batch=2, t_max=4)
    a, b = bench.make_network(cfg, 0), bench.make_network(cfg, 0)
    assert (a["w"] == b["w"]).all() and (a["src"] == b["src"]).all()


def _loss_and_grads(x, w, w_in, target):
    """A small recurrent LIF-like network in plain torch on the CPU (dense
    masked recurrent weights, sigmoid-smoothed spikes): mean squared error of
    a readout of its spikes, and the gradients of the weights."""
    w = w.clone().requires_grad_(True)
    w_in = w_in.clone().requires_grad_(True)
    T, B, _ = x.shape
    n = w.shape[0]
    v = torch.zeros(B, n)
    psc = torch.zeros(B, n)
    zs = []
    for t in range(T):
        v = v + (-v / 20.0 + psc + x[t] @ w_in)
        z = torch.sigmoid(5.0 * (v - 1.0))
        v = v - v.detach() * (z.detach() > 0.5)
        psc = psc * 0.8 + z @ w
        zs.append(z)
    loss = ((torch.stack(zs).mean(-1) - target) ** 2).mean()
    loss.backward()
    return loss.detach(), w.grad, w_in.grad


def _train_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from btorch_b200.replicas import allreduce_gradients

        x, w, w_in, target = _problem()
        half = x.shape[1] // world
        sl = slice(rank * half, (rank + 1) * half)
        _, gw, gw_in = _loss_and_grads(x[:, sl], w, w_in, target[:, sl])
        params = [torch.nn.Parameter(w.clone()), torch.nn.Parameter(w_in.clone())]
        params[0].grad, params[1].grad = gw, gw_in
        nbytes = allreduce_gradients(params)
        out[rank] = (params[0].grad.numpy().copy(), params[1].grad.numpy().copy(), nbytes)
    finally:
        dist.destroy_process_group()


def _problem():
    g = torch.Generator().manual_seed(3)
    n, B, T, c = 48, 8, 12, 10
    w = (torch.rand(n, n, generator=g) < 0.1) * torch.randn(n, n, generator=g) * 0.3
    w_in = torch.randn(c, n, generator=g) * 0.4
    x = (torch.rand(T, B, c, generator=g) < 0.3).float()
    target = torch.rand(T, B, generator=g) * 0.2
    return x, w, w_in, target


def test_two_ranks_allreduced_gradient_equals_the_union_batch_gradient():
    """Data-parallel training step: each of two gloo ranks computes the
    gradient of the mean loss over its half of the batch; one all-reduce of
    the flattened gradients (averaged) gives every rank the gradient of the
    mean loss over the whole batch, as a single process computes it."""
    import numpy as np

    port = 29400 + os.getpid() % 1000
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_train_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    x, w, w_in, target = _problem()
    _, gw, gw_in = _loss_and_grads(x, w, w_in, target)
    for rank in (0, 1):
        np.testing.assert_allclose(res[rank][0], gw.numpy(), rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(res[rank][1], gw_in.numpy(), rtol=1e-5, atol=1e-7)
        assert res[rank][2] == (gw.numel() + gw_in.numel()) * 4
    np.testing.assert_array_equal(res[0][0], res[1][0])


def _replica_events_rank(rank, world, port, out):
    """Each rank runs its own seeded input through the oracle (the same
    network on every rank) and reports through bench.job_totals."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import time

        import bench

        cfg = dict(bench.CONFIGS["connectome"], n=2000, indeg=40, batch=2, t_max=30, dur=(30, 30))
        net = bench.make_network(cfg, 0)
        x, _ = bench.host_inputs(cfg, rank, 30)
        t0 = time.perf_counter()
        e, _, _, _ = bench.cpu_sample(cfg, net, x, 30)
        ms = (time.perf_counter() - t0) * 1e3
        t, tot = bench.job_totals(ms, e, torch.device("cpu"))
        out[rank] = (ms, e, t, tot)
    finally:
        dist.destroy_process_group()


def test_two_replicas_of_real_work_sum_events_and_take_the_slowest_time():
    port = 29600 + os.getpid() % 1000
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_replica_events_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    (ms0, e0, t0, s0), (ms1, e1, t1, s1) = res[0], res[1]
    assert e0 > 0 and e1 > 0 and e0 != e1  # per-rank seeded inputs
    assert s0 == s1 == e0 + e1
    assert t0 == t1 == max(ms0, ms1)
