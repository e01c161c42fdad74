"""bench.py's multi-rank bookkeeping on CPU (gloo, world size 2): replicas'
whole-job throughput uses every rank's points over the slowest rank's time,
and the reference arm prints on rank 0 only."""
import io
import os
import socket
import sys
import contextlib

import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        secs_local = 2.0 + rank           # rank 1 is the slowest
        value, secs = bench.replicas_value(1.0e6, 10, secs_local, world, "cpu")
        out = io.StringIO()

        class Args:
            n, steps, warmup = 16, 1, 0
        if rank != 0:   # the reference arm: ranks other than 0 exit without work or output
            with contextlib.redirect_stdout(out):
                bench.run_reference(Args, rank, world)
        q.put((rank, value, secs, out.getvalue()))
    finally:
        dist.destroy_process_group()


def test_replicas_value_and_reference_arm_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, secs, out in res:
        assert secs == 3.0
        assert abs(value - 2 * 1.0e6 * 10 / 3.0 / 1e6) < 1e-12
    assert res[1][3] == ""
