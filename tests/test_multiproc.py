"""The N > 1 host logic of bench.py on CPU: two gloo ranks.

bench.py runs one replica per GPU and reports all ranks' units over the
slowest rank's time; every rank takes part in the same collectives.  The
reference arm runs on rank 0 alone and the other ranks exit quietly."""
import json
import os
import socket
import subprocess
import sys
from datetime import timedelta

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench

    value, ms = bench.aggregate_throughput(1000.0, 2.0 + rank, world, scale=1.0)  # rank 1 is slower
    slowest = bench.max_over_ranks(5.0 * (rank + 1), world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, value, ms, slowest))


def test_aggregation_takes_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, value, ms, slowest in got:
        assert ms == 3.0  # the slower rank's time, on every rank
        assert abs(value - world * 1000.0 / 3e-3) < 1e-6
        assert slowest == 10.0


def _run_reference(rank, world):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                           "sort", "--steps", "1", "--warmup", "1", "--gpus", str(world)],
                          capture_output=True, text=True, env=env, timeout=300)


def test_reference_arm_runs_on_rank_zero_only():
    r1 = _run_reference(1, 2)
    assert r1.returncode == 0 and r1.stdout.strip() == ""
    r0 = _run_reference(0, 2)
    assert r0.returncode == 0, r0.stderr
    line = json.loads(r0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["n_gpus"] == 2
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
