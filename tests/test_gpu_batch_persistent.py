"""The batch on one persistent kernel (gtob_batch_run_persistent: every
iteration of the spots in flight is one launch whose CTAs take (spot, step,
node tile) tickets from a device work queue) against the same spots solved
one at a time the way the reference's batch report does (solve_quiet,
solve_cli.rs:338-362): identical iteration counts and exploitability, root
EVs, and synced arenas bit for bit -- with spots joining and leaving the
kernel's set as they finish, and every shape the tuner tries."""
import copy

import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAX_IT, TARGET, CHECK = 60, 0.5, 20


def _configs():
    a = W.small_flop_spot()
    b = W.iso_spot()
    c = copy.deepcopy(W.small_flop_spot())
    c["board"] = "KdQc4s"
    d = W.turn_spot(g.evaluate7, seed=2)  # 564 hands a side, river chance nodes and all-in runouts
    return [a, b, c, d]


def _root_ev(spot, gpu, p):
    """solve_cli.rs:176-188 (query.rs:490-600: ev = cfv / valid + put over
    hands with valid > 1e-9, weighted by the range)."""
    c1, c2, w, same = spot.hands(p)
    oc1, oc2, ow, _ = spot.hands(1 - p)
    ow = ow.astype(np.float64)
    s = np.zeros(52)
    np.add.at(s, oc1, ow)
    np.add.at(s, oc2, ow)
    same_r = np.where(same != 0xFFFFFFFF, ow[np.minimum(same, len(ow) - 1)], 0.0)
    valid = ow.sum() - s[c1] - s[c2] + same_r
    cfv = gpu.root_cfv(p, 1).astype(np.float64)
    put = spot.tree()["put0" if p == 0 else "put1"][0]
    ok = valid > 1e-9
    ev = (cfv[ok] / valid[ok] + put).astype(np.float32).astype(np.float64)
    return float((ev * w[ok]).sum() / w[ok].astype(np.float64).sum())


def _solve_quiet(cfg, storage, device_format):
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage=storage, use_iso=True)
    gpu = g.GpuSolver(host, device_format=device_format)
    pot = cfg["tree"]["starting_pot"]
    while True:
        gpu.iterate(1)
        it = gpu.iteration
        if it % CHECK == 0 or it >= MAX_IT:
            pct = gpu.exploitability(host) / pot * 100
            if pct <= TARGET or it >= MAX_IT:
                break
    ev = [_root_ev(spot, gpu, p) for p in (0, 1)]
    gpu.sync_to_cpu(host)
    return host, it, pct, ev


@pytest.mark.parametrize("storage,device_format,window", [("f32", None, 2), ("compressed", "i16sr", 3),
                                                          ("compressed", None, 8)])
def test_persistent_batch_matches_one_spot_at_a_time(tmp_path, monkeypatch, storage, device_format, window):
    monkeypatch.setenv("GTOB_TUNE_CACHE", str(tmp_path / "shapes.txt"))
    cfgs = _configs()
    batch = g.Batch([g.Spot(c) for c in cfgs], storage=storage, use_iso=True, device_format=device_format)
    batch.run(max_iterations=MAX_IT, target_pct=TARGET, check_every=CHECK, persistent=True, window=window)
    rows = batch.rows()
    st = batch.stats()
    assert st["launches"] >= MAX_IT and st["kernel_ms"] > 0 and st["grid"] >= 148, st
    for i, cfg in enumerate(cfgs):
        host, it, pct, ev = _solve_quiet(cfg, storage, device_format)
        r = rows[i]
        assert r["status"] == 0 and r["error"] == "", r
        assert r["iterations"] == it, (i, r, it)
        assert r["exploit_pct"] == pct, (i, r, pct)
        for p in (0, 1):
            assert abs(r["ev"][p] - ev[p]) <= 1e-9 * max(1.0, abs(ev[p])), (i, p, r["ev"], ev)
        bs = batch.solver(i)
        assert bs.iteration == it
        for which in (0, 1):
            for p in (0, 1):
                assert np.array_equal(bs.arena(which, p), host.arena(which, p)), (i, which, p)


def test_persistent_batch_tunes_once_per_size_class(tmp_path, monkeypatch):
    """The first run of a size class times its candidate shapes on real
    iterations and writes the choice; a second run reads it back."""
    cache = tmp_path / "shapes.txt"
    monkeypatch.setenv("GTOB_TUNE_CACHE", str(cache))
    cfgs = [W.turn_spot(g.evaluate7, seed=2)] * 2
    a = g.Batch([g.Spot(c) for c in cfgs], storage="f32", keep_solvers=False)
    a.run(max_iterations=40, target_pct=0.0, check_every=20, persistent=True, window=2)
    sa = a.stats()
    assert sa["tuned"] == 1 and sa["launches"] == 40, sa
    lines = cache.read_text().split()
    assert len(lines) == 4 and int(lines[2]) == sa["tile"], lines
    b = g.Batch([g.Spot(c) for c in cfgs], storage="f32", keep_solvers=False)
    b.run(max_iterations=40, target_pct=0.0, check_every=20, persistent=True, window=2)
    sb = b.stats()
    assert sb["tuned"] == 0 and (sb["tile"], sb["ctas_per_sm"]) == (sa["tile"], sa["ctas_per_sm"]), (sa, sb)
    for ra, rb in zip(a.rows(), b.rows()):
        assert (ra["iterations"], ra["exploit_pct"]) == (rb["iterations"], rb["exploit_pct"])


def test_persistent_batch_keeps_unsupported_spots_in_their_row(tmp_path, monkeypatch):
    """The kernel takes nodes of at most 4 actions: a spot whose root has 5
    fails in its own row, the others solve."""
    monkeypatch.setenv("GTOB_TUNE_CACHE", str(tmp_path / "shapes.txt"))
    wide = copy.deepcopy(W.small_flop_spot())
    for side in ("oop", "ip"):
        wide["tree"][side][0]["bet"] = W.sizes("25", "50", "75", "100")
    cfgs = [W.small_flop_spot(), wide, W.iso_spot()]
    batch = g.Batch([g.Spot(c) for c in cfgs], storage="f32")
    batch.run(max_iterations=20, target_pct=0.0, check_every=10, persistent=True, window=3)
    rows = batch.rows()
    assert rows[1]["status"] != 0 and "4 actions" in rows[1]["error"], rows[1]
    for i in (0, 2):
        assert rows[i]["status"] == 0 and rows[i]["iterations"] == 20, rows[i]
        assert np.isfinite(rows[i]["exploit_pct"])
