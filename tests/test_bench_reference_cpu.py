"""bench.py --impl reference (the CPU algorithm timed on the host cores) keeps
the benchmark line contract: launched under torchrun with two ranks, rank 0
alone prints one JSON line with the headline workload's metric, its CPU
baseline and a zero-copy e2e entry; the other rank exits 0 without work."""

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_two_ranks_prints_one_line():
    port = 29700 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--cpu-sample-steps", "1", "--cpu-events-steps", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == "synaptic_events_per_s" and line["unit"] == "events/s"
    assert line["higher_is_better"] is True and line["n_gpus"] == 2
    assert line["steps"] == 1 and line["warmup"] == 0
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["config"]["workload"].startswith("batched:")
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert "events per live sample-step" in cb["sample"] and "event-driven run of 3 steps" in cb["sample"]
    assert line["neuron_steps_per_s"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "events/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
