"""One spot split over shards (a flop by turn card),
run as every shard of the spot on one GPU with the split subtrees' values
summed on the host between them, against one engine on the whole spot: the
sum is exact (each value is nonzero on one shard), so exploitability and
every arena entry must be identical.  The NCCL form (one process per GPU)
runs here with one rank."""
import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg_fn,use_iso", [(W.small_flop_spot, False), (W.iso_spot, True)])
@pytest.mark.parametrize("nshards,device_format", [(2, "f32"), (3, "f32"), (2, "i16")])
def test_shards_match_one_engine(cfg_fn, use_iso, nshards, device_format):
    cfg = cfg_fn()
    pot = cfg["tree"]["starting_pot"]
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", use_iso=use_iso)
    one = g.GpuSolver(host, device_format=device_format)
    one.iterate(12)
    e1 = one.exploitability(host)
    sh = g.Shards(host, nshards, device_format=device_format)
    sh.iterate(12)
    e2 = sh.exploitability(host)
    assert e1 == e2, (e1, e2, pot)
    for which in (0, 1):
        for p in (0, 1):
            assert np.array_equal(one.export_arena(which, p), sh.export_arena(which, p)), (which, p)


def test_nccl_single_rank_equals_one_engine():
    cfg = W.small_flop_spot()
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", use_iso=False)
    one = g.GpuSolver(host)
    one.iterate(5)
    nid = g.nccl_unique_id()
    assert len(nid) == 128
    sharded = g.sharded_gpu_solver(host, 0, 1, nid)
    sharded.iterate(5)
    assert sharded.exploitability(host) == one.exploitability(host)
    for which in (0, 1):
        for p in (0, 1):
            assert np.array_equal(sharded.export_arena(which, p), one.export_arena(which, p))


@pytest.mark.parametrize("cfg_fn,use_iso,storage", [(W.small_flop_spot, False, "f32"), (W.iso_spot, True, "compressed")])
def test_shards_sync_to_cpu(tmp_path, cfg_fn, use_iso, storage):
    """Every shard synced into one host solver gives the host arenas (and the
    saved file) that one engine's sync gives."""
    spot = g.Spot(cfg_fn())
    ha = g.Solver(spot, storage=storage, use_iso=use_iso)
    hb = g.Solver(spot, storage=storage, use_iso=use_iso)
    one = g.GpuSolver(ha)
    one.iterate(7)
    one.sync_to_cpu(ha)
    sh = g.Shards(hb, 2)
    sh.iterate(7)
    sh.sync_to_cpu(hb)
    for which in (0, 1):
        for p in (0, 1):
            assert np.array_equal(ha.arena(which, p), hb.arena(which, p)), (which, p)
    ha.save(tmp_path / "a.gto")
    hb.save(tmp_path / "b.gto")
    assert (tmp_path / "a.gto").read_bytes() == (tmp_path / "b.gto").read_bytes()
