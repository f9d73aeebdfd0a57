""".gto save and load straight from and into device memory (gtob_gpu_save,
gtob_gpu_load), against the host path they replace.

* Device save: the file must be byte-identical to what the reference's flow
  writes -- GpuSolver::sync_to_cpu into an f32 host solver, then
  Solver::ensure_symmetric and Solver::save (save.rs:92-143) -- including the
  suit-isomorphic branches the device never holds (gathered on the device
  through composed hand permutations) and a lock whose sigma a symmetric
  branch takes as its strategy sums (cfr.rs:806-871).
* Device load: the device state after gtob_gpu_load must equal the state of
  a GPU solver built from Solver::load_with_storage (save.rs:149-227) of the
  same file, arena for arena, and stay equal over further iterations.
"""
import os

import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _solved(cfg, iters, use_iso, device_format, lock):
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", use_iso=use_iso)
    if lock:
        # a turn node below check-check: its suit-mirrored sibling is a
        # symmetric branch that takes the lock's sigma as strategy sums
        host.lock_node([0, 0, "Ah"], "freeze", label="frozen turn node")
    gpu = g.GpuSolver(host, device_format=device_format)
    gpu.iterate(iters)
    return spot, host, gpu


@pytest.mark.parametrize("device_format", ["f32", "i16"])
@pytest.mark.parametrize("case", ["iso", "iso_lock", "no_iso"])
def test_device_save_matches_host_save(tmp_path, device_format, case):
    cfg = W.small_flop_spot() if case == "no_iso" else W.iso_spot()
    spot, host, gpu = _solved(cfg, 7, case != "no_iso", device_format, case == "iso_lock")
    if case != "no_iso":
        assert gpu.info()["visited_nodes"] < spot.num_nodes  # symmetric branches exist
    before = host.arena(1, 0).copy()
    pa, pb = tmp_path / "dev.gto", tmp_path / "host.gto"
    gpu.save(pa, host)
    assert np.array_equal(host.arena(1, 0), before)  # the host solver is not touched
    assert not os.path.exists(str(pa) + ".tmp")
    gpu.sync_to_cpu(host)
    host.ensure_symmetric()
    host.save(pb)
    a, b = pa.read_bytes(), pb.read_bytes()
    assert len(a) == len(b)
    assert a == b


@pytest.mark.parametrize("device_format", ["f32", "i16"])
def test_device_load_matches_host_load(tmp_path, device_format):
    cfg = W.iso_spot()
    spot, host, gpu = _solved(cfg, 9, True, device_format, True)
    path = tmp_path / "s.gto"
    gpu.save(path, host)
    gpu.close()
    h_host = g.Solver.load(path, storage="f32")
    ga = g.GpuSolver(h_host, device_format=device_format)
    h_dev, gb = g.GpuSolver.load(path, storage="f32", device_format=device_format)
    assert gb.iteration == ga.iteration == 9
    assert h_dev.num_locks == h_host.num_locks == 1
    for rounds in range(2):
        for which in (0, 1):
            for p in (0, 1):
                assert np.array_equal(ga.export_arena(which, p), gb.export_arena(which, p)), (rounds, which, p)
        ga.iterate(4)
        gb.iterate(4)
    assert ga.exploitability(h_host) == gb.exploitability(h_dev)
    gb.sync_to_cpu(h_dev)
    ga.sync_to_cpu(h_host)
    for which in (0, 1):
        for p in (0, 1):
            assert np.array_equal(h_dev.arena(which, p), h_host.arena(which, p))


def test_device_save_then_load_round_trip(tmp_path):
    """A device save loaded back onto the device gives the saved device
    blocks back exactly (f32 arenas)."""
    spot, host, gpu = _solved(W.small_flop_spot(), 6, False, "f32", False)
    path = tmp_path / "r.gto"
    gpu.save(path, host)
    h2, g2 = g.GpuSolver.load(path, device_format="f32")
    for which in (0, 1):
        for p in (0, 1):
            assert np.array_equal(gpu.export_arena(which, p), g2.export_arena(which, p))


def test_device_save_refuses_another_spot(tmp_path):
    spot, host, gpu = _solved(W.small_flop_spot(), 1, False, "f32", False)
    other = g.Solver(g.Spot(W.iso_spot()))
    with pytest.raises(g.GtobError) as e:
        gpu.save(tmp_path / "x.gto", other)
    assert "not the one" in str(e.value)
    assert not os.path.exists(tmp_path / "x.gto")


@pytest.mark.parametrize("device_format,algo", [("fp8", "dcfr"), ("f32", "pcfr+"), ("i16", "pcfr+")])
def test_device_save_load_other_formats(tmp_path, device_format, algo):
    """FP8 arenas and PCFR+ (whose predictions the format does not hold):
    the device save equals the host path's file, and a device load equals a
    host load + GpuSolver (predictions restart at zero in both)."""
    cfg = W.small_flop_spot()
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", algo=algo, use_iso=False)
    gpu = g.GpuSolver(host, device_format=device_format)
    gpu.iterate(6)
    pa, pb = tmp_path / "dev.gto", tmp_path / "host.gto"
    gpu.save(pa, host)
    gpu.sync_to_cpu(host)
    host.ensure_symmetric()
    host.save(pb)
    assert pa.read_bytes() == pb.read_bytes()
    h_host = g.Solver.load(pb, storage="f32")
    ga = g.GpuSolver(h_host, device_format=device_format)
    h_dev, gb = g.GpuSolver.load(pa, storage="f32", device_format=device_format)
    for which in (0, 1):
        for p in (0, 1):
            assert np.array_equal(ga.export_arena(which, p), gb.export_arena(which, p)), (which, p)
    ga.iterate(3)
    gb.iterate(3)
    assert ga.exploitability(h_host) == gb.exploitability(h_dev)
