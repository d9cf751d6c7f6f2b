"""The N > 1 path of bench.py on CPU: two ranks on the gloo backend. Each GPU
runs an independent replica (the path does not shard), so ranks meet only at
barriers and the maximum-over-ranks reduction of their timings; the
whole-job rate counts every rank's units over the slowest rank's time, and the
reference arm runs on rank 0 alone."""
import datetime
import io
import os
import socket
import sys
import contextlib

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        timings = bench.max_over_ranks([10.0 + rank, 5.0 - rank, float(rank)])
        rate = bench.whole_job_rate(1000, world, timings[0])
        out = io.StringIO()
        with contextlib.redirect_stdout(out):
            if rank != 0:
                bench.run_reference(None, rank)  # ranks other than 0 return at once
        dist.barrier()
        q.put((rank, timings, rate, out.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_their_timings():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, timings, rate, printed in results:
        assert timings == [11.0, 5.0, 1.0]  # element-wise maximum over the two ranks
        assert abs(rate - 2 * 1000 / 11e-3) < 1e-6 * rate
        assert printed == ""


def test_single_process_helpers():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.0, 4.5]) == [3.0, 4.5]
    assert bench.whole_job_rate(500, 1, 250.0) == 2000.0
