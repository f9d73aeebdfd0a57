"""bench.py's multi-rank plumbing on CPU: two gloo ranks (127.0.0.1), as
torchrun would launch them.  Each rank times its own replica; the reported
time is the max over ranks, and the reference arm prints from rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    try:
        w, r, _ = bench.dist_setup(world, backend="gloo")
        assert (w, r) == (world, rank)
        bench.barrier(w)
        got = bench.allmax(10.0 + 5.0 * rank, w)
        # the reference arm: only rank 0 works and prints
        buf = io.StringIO()

        class A:
            pass
        a = A()
        a.workload, a.steps, a.warmup, a.storage, a.cpu_threads, a.gpus = "river", 1, 0, "f32", 1, world
        if rank != 0:
            with redirect_stdout(buf):
                bench.run_reference(a, w, r)
        q.put((rank, got, buf.getvalue()))
        bench.barrier(w)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_and_rank0_only():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[1] for r in res] == [15.0, 15.0]  # max over ranks
    assert res[1][2] == ""  # rank 1 of the reference arm prints nothing
