"""Batch of spots on one GPU (gtob_batch_*) against the same spots solved one
at a time the way the reference's batch report does (solve_quiet,
solve_cli.rs:338-362): identical iteration counts, exploitability and synced
arenas, root EVs as solve_cli.rs:176-188 computes them, and a failing spot
that leaves the others solving."""
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
    return [a, b, c]


def _root_ev(spot, gpu, p):
    """solve_cli.rs:176-188: reach-weighted average of the root EVs
    (query.rs:490-600, ev = cfv / valid + put, hands with valid > 1e-9)."""
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


def _solve_quiet(cfg):
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", use_iso=True)
    gpu = g.GpuSolver(host)
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
    return spot, host, it, pct, ev


def test_batch_matches_one_spot_at_a_time():
    cfgs = _configs()
    batch = g.Batch([g.Spot(c) for c in cfgs], storage="f32", use_iso=True)
    batch.run(max_iterations=MAX_IT, target_pct=TARGET, check_every=CHECK, workers=3)
    rows = batch.rows()
    for i, cfg in enumerate(cfgs):
        spot, host, it, pct, ev = _solve_quiet(cfg)
        r = rows[i]
        assert r["status"] == 0 and r["error"] == "", r
        assert r["iterations"] == it
        assert r["exploit_pct"] == pct
        assert r["seconds"] > 0
        for p in (0, 1):
            assert abs(r["ev"][p] - ev[p]) <= 1e-9 * max(1.0, abs(ev[p])), (i, p, r["ev"], ev)
        bs = batch.solver(i)
        assert bs.iteration == it
        for which in (0, 1):
            for p in (0, 1):
                assert np.array_equal(bs.arena(which, p), host.arena(which, p)), (i, which, p)


def test_batch_keeps_failures_in_their_row():
    """FP8 arenas take nodes of at most 4 actions: a spot whose root has 5
    fails in its own row, the others solve."""
    wide = copy.deepcopy(W.small_flop_spot())
    for side in ("oop", "ip"):
        wide["tree"][side][0]["bet"] = W.sizes("25", "50", "75", "100")
    cfgs = [W.small_flop_spot(), wide, W.iso_spot()]
    batch = g.Batch([g.Spot(c) for c in cfgs], device_format="fp8")
    batch.run(max_iterations=20, target_pct=0.0, check_every=10, workers=2)
    rows = batch.rows()
    assert rows[1]["status"] == -1 and "4 actions" in rows[1]["error"], rows[1]
    for i in (0, 2):
        assert rows[i]["status"] == 0 and rows[i]["iterations"] == 20, rows[i]
        assert np.isfinite(rows[i]["exploit_pct"])


def test_batch_without_solvers_gives_the_same_rows():
    """A batch that keeps no host solvers (the report mode: each worker solves
    against a solver without arenas) reports the same rows."""
    cfgs = _configs()
    spots = [g.Spot(c) for c in cfgs]
    kept = g.Batch(spots, storage="f32", use_iso=True)
    kept.run(max_iterations=MAX_IT, target_pct=TARGET, check_every=CHECK, workers=2)
    lean = g.Batch(spots, storage="f32", use_iso=True, keep_solvers=False)
    lean.run(max_iterations=MAX_IT, target_pct=TARGET, check_every=CHECK, workers=3)
    for a, b in zip(kept.rows(), lean.rows()):
        assert (a["status"], a["iterations"], a["exploit_pct"], a["ev"]) == \
               (b["status"], b["iterations"], b["exploit_pct"], b["ev"])
    with pytest.raises(IndexError):
        lean.solver(0)
