"""The benchmark configurations themselves on the GPU engine against the CPU
oracle (no pruning, exact terminal sums -- the level-synchronous sweep's
arithmetic), at the iteration counts the configurations name:

* river (c1): all 1081 combos a side, f32 arenas, 500 DCFR iterations;
* turn (c2): 564 v 564, 1000 DCFR iterations with f32 arenas, with i16/u16
  (store.rs rounding) and with i16/u16 under stochastic rounding;
* flop (c3, the default bench workload): 10,835,022 nodes, 470 v 647 hands,
  i16/u16 arenas with stochastic rounding (the bench's format), 5 DCFR
  iterations (the oracle's unpruned iteration of this tree takes seconds on
  the host cores).

Bars: exploitability within 0.01% of the pot; average strategies within 1e-4
absolute (every action node on c1/c2, a seeded sample of 12,000 action nodes on
c3); on c1/c2 also the count of arena entries that differ from the oracle's
bits, which is expected to be zero.
"""
import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

STRAT_TOL = 1e-4
EXPL_TOL_PCT = 0.01


def _sigma(s, off, na, nh):
    blk = np.maximum(s[off:off + na * nh].reshape(na, nh).astype(np.float64), 0.0)
    tot = blk.sum(0)
    return np.where(tot > 1e-12, blk / np.where(tot > 0, tot, 1.0), 1.0 / na)


def _worst_strategy(spot, host, osv, nodes_by_player):
    t = spot.tree()
    worst = 0.0
    for p in (0, 1):
        a, b = host.arena(1, p), osv.arena(1, p)
        nh = spot.nh[p]
        for n in nodes_by_player[p]:
            na, off = int(t["nchild"][n]), int(t["data_off"][n])
            worst = max(worst, float(np.abs(_sigma(a, off, na, nh) - _sigma(b, off, na, nh)).max()))
    return worst


def _action_nodes(spot):
    t = spot.tree()
    return {p: np.nonzero((t["kind"] == 0) & (t["player"] == p))[0] for p in (0, 1)}


@pytest.mark.parametrize("name,cfg_fn,iters,storage", [
    ("c1 river", lambda: W.river_spot(seed=1), 500, "f32"),
    ("c2 turn", lambda: W.turn_spot(g.evaluate7, seed=2), 1000, "f32"),
    ("c2 turn", lambda: W.turn_spot(g.evaluate7, seed=2), 1000, "compressed"),
    ("c2 turn", lambda: W.turn_spot(g.evaluate7, seed=2), 1000, "i16sr"),
])
def test_config_full_length_matches_oracle(name, cfg_fn, iters, storage):
    cfg = cfg_fn()
    pot = cfg["tree"]["starting_pot"]
    sr = storage == "i16sr"
    ospot = po.Spot(cfg)
    osv = po.Solver(ospot, compressed=storage != "f32", algo="dcfr", use_iso=True, prune=False, exact=True,
                    stochastic=sr)
    osv.iterate(iters)
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="compressed" if sr else storage, algo="dcfr", use_iso=True)
    gpu = g.GpuSolver(host, device_format="i16sr" if sr else None)
    gpu.iterate(iters)
    eg = gpu.exploitability(host)
    gpu.sync_to_cpu(host)
    host.ensure_symmetric()
    osv.ensure_symmetric()
    eo = osv.exploitability()
    assert abs(eg - eo) / pot * 100 < EXPL_TOL_PCT, (name, storage, eg, eo)
    worst = _worst_strategy(spot, host, osv, _action_nodes(spot))
    assert worst < STRAT_TOL, (name, storage, worst)
    diff = sum(int(np.count_nonzero(host.arena(w, p) != osv.arena(w, p))) for w in (0, 1) for p in (0, 1))
    assert diff == 0, (name, storage, "arena entries differing from the oracle", diff)


def test_flop_config_matches_oracle():
    """The headline flop (seed 3, i16/u16 with stochastic rounding), 5
    iterations of the staged engine against 5 of the oracle."""
    cfg = W.flop_spot(g.evaluate7, seed=3)
    pot = cfg["tree"]["starting_pot"]
    iters = 5
    ospot = po.Spot(cfg)
    osv = po.Solver(ospot, compressed=True, algo="dcfr", use_iso=True, prune=False, exact=True, stochastic=True)
    osv.iterate(iters)
    eo = osv.exploitability()
    spot = g.Spot(cfg)
    assert spot.num_nodes == 10835022 and tuple(spot.nh) == (470, 647)
    host = g.Solver(spot, storage="compressed", algo="dcfr", use_iso=True)
    gpu = g.GpuSolver(host, device_format="i16sr")
    gpu.iterate(iters)
    eg = gpu.exploitability(host)
    assert abs(eg - eo) / pot * 100 < EXPL_TOL_PCT, (eg, eo)
    gpu.sync_to_cpu(host)
    gpu.close()
    # a seeded sample of action nodes that the solve reached (a non-zero
    # strategy-sum block on the oracle's side)
    nodes = _action_nodes(spot)
    t = spot.tree()
    rng = np.random.default_rng(2026)
    sample = {}
    for p in (0, 1):
        s = osv.arena(1, p)
        nh = spot.nh[p]
        cand = rng.choice(nodes[p], size=min(20000, len(nodes[p])), replace=False)
        live = [n for n in cand
                if np.any(s[int(t["data_off"][n]):int(t["data_off"][n]) + int(t["nchild"][n]) * nh] != 0)]
        sample[p] = live[:6000]
    assert sum(len(v) for v in sample.values()) >= 10000
    worst = _worst_strategy(spot, host, osv, sample)
    assert worst < STRAT_TOL, worst
