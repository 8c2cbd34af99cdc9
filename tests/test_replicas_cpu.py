"""The multi-GPU path is replicas only: every rank runs its own simulation and
the job's throughput is all ranks' particle-steps over the slowest rank's
device time. These tests run that aggregation as two gloo ranks on the CPU
(the same calls bench.py makes over NCCL), and check that only rank 0 of the
reference arm does work."""
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


def _rank(rank, ws, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    own_ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
    m = bench.rank_max(dist, own_ms, "cpu")
    v = bench.job_value(1000 * 10, ws, m)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, m, v))


def test_two_replicas_take_the_slowest_rank():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for rank, m, v in res:
        assert m == 150.0                       # both ranks see the slowest time
        assert v == pytest.approx(1000 * 10 * 2 / 0.150)



def test_reference_arm_other_ranks_do_nothing(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps = 1
        warmup = 0
        workload = "disk512k"
        theta = None

    assert bench.run_reference(A(), 2, 1, 1) is None
    assert capsys.readouterr().out == ""
