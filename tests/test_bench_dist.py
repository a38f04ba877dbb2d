"""Host logic of bench.py's multi-rank (replica) path, run as two gloo ranks on the CPU: the
reported time is the max over ranks and the value aggregates all replicas."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local_ms = 1000.0 + 250.0 * rank  # rank 1 is slower
    t = bench.max_over_ranks(local_ms, dist, "cpu")
    v = bench.whole_job_tflops(world, 3, 16384, t)
    q.put((rank, t, v))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_max_over_ranks():
    import bench
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, v in res:
        assert t == pytest.approx(1250.0)
        assert v == pytest.approx(bench.whole_job_tflops(2, 3, 16384, 1250.0))
    assert bench.whole_job_tflops(2, 3, 16384, 1250.0) == pytest.approx(
        2 * bench.whole_job_tflops(1, 3, 16384, 1250.0))
