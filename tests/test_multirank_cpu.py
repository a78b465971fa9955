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
