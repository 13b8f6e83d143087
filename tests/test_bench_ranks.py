"""The multi-rank (replicas) logic of bench.py on CPU: two gloo ranks with
different step times report the slowest rank's time and the whole-job value;
rank 1 of the reference arm does no work."""
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


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, device="cpu")
    value = bench.whole_job_tflops(2e12, world, ms)
    ref = bench.reference_arm(type("A", (), {"size": 8, "trans_a": 0, "steps": 1, "warmup": 0,
                                             "gpus": world})(), world, 1) if rank == 1 else None
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, value, ref))


def test_two_gloo_ranks_report_max_time_and_total_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value, ref in out:
        assert ms == pytest.approx(15.0)
        assert value == pytest.approx(2 * 2e12 / 15e-3 / 1e12)
    assert out[1][3] is None
