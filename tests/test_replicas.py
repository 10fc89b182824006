"""The N > 1 path of bench.py: N independent replicas, one process per GPU.
Here as two gloo ranks on the CPU: the whole-job figures take each time
from the slowest rank and sum the work of all ranks, and the reference arm
runs on rank 0 only."""
import datetime
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        times = [[4.0, 9.0, 1.5], [6.0, 2.0, 1.0]][rank]
        updates = [[100.0, 50.0, 10.0], [300.0, 70.0, 20.0]][rank]
        t, u = bench.aggregate_replicas(times, updates, dist, "cpu")
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, t, u))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), None))


def test_replica_aggregation_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, u in out:
        assert u is not None, t
        assert t == [6.0, 9.0, 1.5]
        assert u == [400.0, 120.0, 30.0]


def test_single_process_aggregation_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate_replicas([1.0, 2.0], [3.0, 4.0]) == ([1.0, 2.0], [3.0, 4.0])


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench
    args = bench.argparse.Namespace(workload="config1", cpu_iters=2, warmup=0, steps=1, gpus=2)
    bench.run_reference(args, rank=1)
    assert capsys.readouterr().out == ""


@pytest.mark.parametrize("rank", [0])
def test_reference_arm_prints_one_line_on_rank_zero(capsys, rank):
    sys.path.insert(0, ROOT)
    import json
    import bench
    args = bench.argparse.Namespace(workload="config1", cpu_iters=2, warmup=0, steps=1, gpus=2)
    bench.run_reference(args, rank=rank)
    lines = [x for x in capsys.readouterr().out.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["cpu_baseline"]["kind"] == "port" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
