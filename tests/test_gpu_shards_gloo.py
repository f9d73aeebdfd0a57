"""One spot split over two processes, each driving one shard on the GPU and
summing the split subtrees' values with torch.distributed.all_reduce over a
gloo group on the host between launches (gtob_gpu_new_sharded_host): the
cross-process form of the sharded solve, which NCCL runs between GPUs.  No
kernel waits on the other rank (each exchange is a host call between two
levels), so both ranks may share one GPU.

Each value is nonzero on exactly one rank, so the f32 sum is exact: both
ranks must report the exploitability one engine reports, bit for bit, and
every arena block a rank holds must equal one engine's block."""
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ITERS = 12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, case, out):
    import datetime

    import torch
    import torch.distributed as dist

    import gtopen_b200 as g
    from gtopen_b200 import workloads as W
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        cfg_name, use_iso, fmt = case
        cfg = W.iso_spot() if cfg_name == "iso" else W.small_flop_spot()
        spot = g.Spot(cfg)
        calls = [0]

        def reduce(values):
            calls[0] += 1
            dist.all_reduce(torch.from_numpy(values))

        host = g.Solver(spot, storage="f32", use_iso=use_iso)
        sh = g.sharded_gpu_solver_host(host, rank, world, reduce, device_format=fmt)
        sh.iterate(ITERS)
        e_sh = sh.exploitability(host)
        arenas = [sh.export_arena(w, p) for w in (0, 1) for p in (0, 1)]
        sh.close()
        # one engine on the whole spot, in this process
        one = g.GpuSolver(g.Solver(spot, storage="f32", use_iso=use_iso), device_format=fmt)
        one.iterate(ITERS)
        e_one = one.exploitability()
        ref = [one.export_arena(w, p) for w in (0, 1) for p in (0, 1)]
        one.close()
        # the blocks of the action nodes this rank's plan visits
        vis = g.shard_visited(spot, rank, world, use_iso).astype(bool)
        t = spot.tree()
        bad, held = 0, 0
        for k, (w, p) in enumerate((w, p) for w in (0, 1) for p in (0, 1)):
            nh = spot.nh[p]
            for n in np.nonzero(vis & (t["kind"] == 0) & (t["player"] == p))[0]:
                lo = int(t["data_off"][n])
                hi = lo + int(t["nchild"][n]) * nh
                held += 1
                bad += int(not np.array_equal(arenas[k][lo:hi], ref[k][lo:hi]))
        out.put((rank, e_sh, e_one, held, bad, calls[0]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", [("small", False, "f32"), ("iso", True, "i16")])
def test_two_processes_match_one_engine(case):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, case, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=600) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, e_sh, e_one, held, bad, calls in res:
        assert e_sh == e_one, (rank, e_sh, e_one)
        assert held > 0 and bad == 0, (rank, held, bad)
        assert calls > 0  # the values did cross between the processes
    assert res[0][1] == res[1][1]
