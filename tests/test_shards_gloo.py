"""The sharded spot's host side with one process per rank (gloo, world size
2, CPU): each rank builds only its own shard's plan, as a rank of a sharded
solve over NCCL does, and the ranks' visit masks, summed with all_reduce,
must cover the tree once below the shared top part and twice inside it."""
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import gtopen_b200 as g
from gtopen_b200 import workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, use_iso, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        spot = g.Spot(W.iso_spot() if use_iso else W.small_flop_spot())
        mine = torch.from_numpy(g.shard_visited(spot, rank, world, use_iso).astype(np.int32))
        count = mine.clone()
        dist.all_reduce(count)
        both = mine.clone()
        dist.all_reduce(both, op=dist.ReduceOp.MIN)  # the top part every rank holds
        if rank == 0:
            full = g.shard_visited(spot, 0, 1, use_iso).astype(np.int32)
            out.put((full.tolist(), count.tolist(), both.tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(use_iso):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, use_iso, q)) for r in range(2)]
    for p in procs:
        p.start()
    full, count, both = (np.array(x) for x in q.get(timeout=300))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return full, count, both


def test_two_ranks_partition_the_spot():
    for use_iso in (False, True):
        full, count, both = _run(use_iso)
        top = both.astype(bool)
        assert np.array_equal(count > 0, full.astype(bool))
        assert np.all(count[top] == 2)
        below = full.astype(bool) & ~top
        assert below.any() and np.all(count[below] == 1)
