"""GPU engine vs the CPU oracle, through the C ABI (libgtob).

The oracle runs the reference CPU engine's arithmetic with zero-reach pruning
off, which is the level-synchronous sweep's semantics (the reference's own GPU
tests note the pruning difference, tests/gpu.rs:67-69), and with the engine's
exact terminal sums (pyoracle exact=True: the fold and showdown reach sums of
game.rs:470-577 taken exactly, so their order does not matter).  Bars:
average strategies within 1e-4 absolute after N iterations, regrets within
1e-4 relative to the arena scale, exploitability within 0.01% of the pot;
with exact sums the arenas are expected to be bit-identical, and
test_arenas_bit_identical holds every engine to that.
"""
import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

STRAT_TOL = 1e-4      # absolute, average strategy
EXPL_TOL_PCT = 0.01   # % of pot


def _avg_strategies(spot, arena_fn):
    """Average strategy per action node from a strategy-sum arena (cfr.rs:679-726)."""
    t = spot.tree()
    out = {}
    for p in (0, 1):
        s = arena_fn(p)
        nh = spot.nh[p]
        for n in np.nonzero((t["kind"] == 0) & (t["player"] == p))[0]:
            na = int(t["nchild"][n])
            off = int(t["data_off"][n])
            blk = np.maximum(s[off:off + na * nh].reshape(na, nh).astype(np.float64), 0.0)
            tot = blk.sum(0)
            sig = np.where(tot > 1e-12, blk / np.where(tot > 0, tot, 1.0), 1.0 / na)
            out[int(n)] = sig
    return out


def _run_pair(cfg, iters, storage="f32", algo="dcfr", use_iso=False, engine="fused"):
    """storage: "f32", "compressed" (i16/u16, store.rs rounding) or "i16sr"
    (i16/u16 requantised with stochastic rounding)."""
    sr = storage == "i16sr"
    ospot = po.Spot(cfg)
    osv = po.Solver(ospot, compressed=storage != "f32", algo=algo, use_iso=use_iso, prune=False, exact=True,
                    stochastic=sr)
    osv.iterate(iters)
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="compressed" if sr else storage, algo=algo, use_iso=use_iso)
    gpu = g.GpuSolver(host, engine=engine, device_format="i16sr" if sr else None)
    gpu.iterate(iters)
    gpu.sync_to_cpu(host)
    return ospot, osv, spot, host, gpu


def _compare(spot, osv, host, what):
    so = _avg_strategies(spot, lambda p: osv.arena(1, p))
    sg = _avg_strategies(spot, lambda p: host.arena(1, p))
    worst = max(float(np.abs(so[n] - sg[n]).max()) for n in so)
    assert worst < STRAT_TOL, "%s: average strategy differs by %g" % (what, worst)
    for p in (0, 1):
        ro, rg = osv.arena(0, p), host.arena(0, p)
        scale = max(1.0, float(np.abs(ro).max()))
        d = float(np.abs(ro - rg).max())
        assert d <= 1e-4 * scale, "%s: regrets[%d] differ by %g (scale %g)" % (what, p, d, scale)


@pytest.mark.parametrize("engine", ["fused", "plain", "warp", "staged"])
@pytest.mark.parametrize("name,cfg_fn,iters", [
    ("clairvoyance", W.clairvoyance_spot, 50),
    ("small_flop", W.small_flop_spot, 20),
    ("river_1081", W.river_spot, 20),
])
def test_f32_dcfr_matches_oracle(name, cfg_fn, iters, engine):
    cfg = cfg_fn()
    ospot, osv, spot, host, gpu = _run_pair(cfg, iters, engine=engine)
    assert host.iteration == iters
    _compare(spot, osv, host, name)
    pot = cfg["tree"]["starting_pot"]
    eo = osv.exploitability()
    eg = gpu.exploitability(host)
    assert abs(eo - eg) / pot * 100 < EXPL_TOL_PCT, (eo, eg)


@pytest.mark.parametrize("engine", ["fused", "plain", "warp", "staged"])
def test_turn_config_f32_and_i16(engine):
    cfg = W.turn_spot(g.evaluate7)
    for storage in ("f32", "compressed"):
        ospot, osv, spot, host, gpu = _run_pair(cfg, 10, storage=storage, engine=engine)
        _compare(spot, osv, host, "turn/" + storage)
        eo, eg = osv.exploitability(), gpu.exploitability(host)
        assert abs(eo - eg) / 100.0 * 100 < EXPL_TOL_PCT, (storage, eo, eg)


@pytest.mark.parametrize("engine", ["fused", "warp", "staged"])
@pytest.mark.parametrize("algo", ["cfr+", "pcfr+"])
@pytest.mark.parametrize("storage", ["f32", "compressed"])
def test_cfrplus_pcfrplus_match_oracle(algo, storage, engine):
    cfg = W.small_flop_spot()
    ospot, osv, spot, host, gpu = _run_pair(cfg, 15, storage=storage, algo=algo, engine=engine)
    _compare(spot, osv, host, "%s/%s" % (algo, storage))


@pytest.mark.parametrize("name,cfg_fn,iters", [
    ("river_1081", W.river_spot, 20),
])
def test_fused32_exploitability_matches_oracle(name, cfg_fn, iters):
    """f32 terminal sums (the reference GPU kernels' precision) round near-tied
    regrets differently from the CPU engine's f64 sums: on the small flop
    fixture that drift exceeds the 0.01%-of-pot bar after 20 iterations,
    which is why the default engines sum terminals exactly.  On the river
    spot the exploitability still agrees with the reference's f64 sums."""
    cfg = cfg_fn()
    ospot = po.Spot(cfg)
    osv = po.Solver(ospot, compressed=False, use_iso=False, prune=False)  # the reference's f64 sums
    osv.iterate(iters)
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", use_iso=False)
    gpu = g.GpuSolver(host, engine="fused32")
    gpu.iterate(iters)
    pot = cfg["tree"]["starting_pot"]
    assert abs(osv.exploitability() - gpu.exploitability(host)) / pot * 100 < EXPL_TOL_PCT


@pytest.mark.parametrize("engine", ["fused", "plain", "warp", "staged"])
@pytest.mark.parametrize("storage,algo", [("f32", "dcfr"), ("compressed", "dcfr"), ("f32", "pcfr+"),
                                          ("compressed", "cfr+"), ("i16sr", "dcfr"), ("i16sr", "pcfr+")])
def test_arenas_bit_identical(engine, storage, algo):
    """With exact terminal sums every engine's regrets and strategy sums equal
    the oracle's bit for bit (16-bit arenas: every quant and scale, as store.rs
    requantises them, or with the stochastic rounding both sides draw from
    the same hash), on a flop spot with folds, showdowns and both chance
    levels, and on an all-in runout spot."""
    cfgs = [W.small_flop_spot()]
    r = W.small_flop_spot()
    for st in r["tree"]["oop"] + r["tree"]["ip"]:
        st["bet"] = [{"PotPct": 75.0}, "AllIn"]
        st["raise"] = ["AllIn"]
    r["tree"]["effective_stack"] = 120.0
    cfgs.append(r)
    for k, cfg in enumerate(cfgs):
        ospot, osv, spot, host, gpu = _run_pair(cfg, 12, storage=storage, algo=algo, engine=engine)
        for p in (0, 1):
            for which in (0, 1):
                a, b = osv.arena(which, p), host.arena(which, p)
                neq = int(np.count_nonzero(a != b))
                assert neq == 0, (k, which, p, neq, a.size, float(np.abs(a - b).max()))


@pytest.mark.parametrize("engine", ["fused", "plain", "warp", "staged"])
def test_iso_matches_oracle(engine):
    cfg = W.iso_spot()
    ospot, osv, spot, host, gpu = _run_pair(cfg, 10, use_iso=True, engine=engine)
    assert spot.num_suit_perms == 2
    _compare(spot, osv, host, "iso")
    eo, eg = osv.exploitability(), gpu.exploitability(host)
    assert abs(eo - eg) / 60.0 * 100 < EXPL_TOL_PCT


def test_device_discounts_bit_exact():
    """DCFR weights computed on the device in f64 equal cfr.rs:44-64 cast to f32."""
    spot = g.Spot(W.clairvoyance_spot())
    for algo in ("dcfr", "cfr+"):
        host = g.Solver(spot, algo=algo)
        gpu = g.GpuSolver(host)
        for t in range(1, 301):
            gpu.iterate(1)
            d = gpu.discounts()
            ref = po.discounts(algo, t)
            assert tuple(np.float32(x) for x in d) == tuple(np.float32(x) for x in ref), (algo, t, d, ref)


def test_clairvoyance_closed_form():
    """tests/gpu.rs:282-335: nuts bet > 0.97, air bluff 0.5 +- 0.05, call 0.5 +- 0.07, < 0.1% pot."""
    spot = g.Spot(W.clairvoyance_spot())
    host = g.Solver(spot, use_iso=False)
    gpu = g.GpuSolver(host)
    gpu.iterate(3000)
    gpu.sync_to_cpu(host)
    e = gpu.exploitability(host)
    assert e / 100.0 * 100 < 0.10
    c1, c2, w, _ = spot.hands(0)
    names = [W.combo_str(int(a), int(b)) for a, b in zip(c1, c2)]
    nuts, air = names.index("AcKc"), names.index("8h7h")
    sig = host.average_strategy(0)
    nh = spot.nh[0]
    assert sig[nh + nuts] > 0.97
    assert abs(sig[nh + air] - 0.5) < 0.05
    t = spot.tree()
    bet_child = int(spot.children()[t["child_start"][0] + 1])
    sig_ip = host.average_strategy(bet_child)
    assert abs(sig_ip[1 * spot.nh[1] + 0] - 0.5) < 0.07


def test_locked_always_call_kills_bluffs():
    """tests/gpu.rs:79-129 on the GPU path."""
    cfg = W.clairvoyance_spot()
    spot = g.Spot(cfg)
    host = g.Solver(spot, use_iso=False)
    gpu = g.GpuSolver(host)
    gpu.iterate(200)
    gpu.sync_to_cpu(host)
    host.lock_node([1], "range", freqs=[0.0, 1.0], label="ip always calls")
    gpu.update_locks(host)
    gpu.iterate(2000)
    gpu.sync_to_cpu(host)
    c1, c2, _, _ = spot.hands(0)
    names = [W.combo_str(int(a), int(b)) for a, b in zip(c1, c2)]
    sig = host.average_strategy(0)
    nh = spot.nh[0]
    assert sig[nh + names.index("AcKc")] > 0.97
    assert sig[nh + names.index("8h7h")] < 0.05


@pytest.mark.parametrize("engine", ["fused", "plain", "warp", "staged"])
def test_exploitability_with_rake_matches_oracle(engine):
    cfg = W.small_flop_spot()
    cfg["tree"]["rake_pct"] = 0.05
    cfg["tree"]["rake_cap"] = 3.0
    ospot, osv, spot, host, gpu = _run_pair(cfg, 30, engine=engine)
    eo, eg = osv.exploitability(), gpu.exploitability(host)
    assert abs(eo - eg) / 60.0 * 100 < EXPL_TOL_PCT, (eo, eg)


def test_root_br_cfv_matches_oracle():
    cfg = W.small_flop_spot()
    ospot, osv, spot, host, gpu = _run_pair(cfg, 25)
    for p in (0, 1):
        a = osv.root_br_cfv(p)
        b = gpu.root_cfv(p, 0)
        assert np.allclose(a, b, rtol=1e-5, atol=1e-4), float(np.abs(a - b).max())


def test_profile_counts_launches():
    spot = g.Spot(W.small_flop_spot())
    host = g.Solver(spot)
    for engine in ("fused", "plain", "warp", "staged"):
        gpu = g.GpuSolver(host, engine=engine)
        pr = gpu.iterate_profiled()
        assert pr.launches[0] == 2 and sum(pr.launches) > 10
        assert gpu.iteration == 1
        if engine == "fused":
            assert pr.launches[3] == 0 and pr.launches[4] == 0  # terminals evaluated in place
        if engine in ("warp", "staged"):
            assert pr.launches[3] == 0 and pr.launches[4] > 0  # folds in place, showdowns launched


def test_allin_runout_spot_matches_oracle():
    """A flop spot with all-in lines: turn and river runout chance nodes whose
    showdown children the fused engine evaluates inside the chance kernel."""
    cfg = W.small_flop_spot()
    for st in cfg["tree"]["oop"] + cfg["tree"]["ip"]:
        st["bet"] = [{"PotPct": 75.0}, "AllIn"]
        st["raise"] = ["AllIn"]
    cfg["tree"]["effective_stack"] = 120.0
    for engine in ("fused", "plain", "warp", "staged"):
        for storage in ("f32", "compressed"):
            ospot, osv, spot, host, gpu = _run_pair(cfg, 12, storage=storage, engine=engine)
            _compare(spot, osv, host, "runout/%s/%s" % (engine, storage))


@pytest.mark.parametrize("engine", ["fused", "plain", "warp", "staged"])
def test_locks_match_oracle(engine):
    """query.rs:700-773 locks on the device path: a frozen root and a
    range-wide lock one step down play their fixed strategies and are never
    updated; every other node matches the oracle."""
    cfg = W.small_flop_spot()
    ospot = po.Spot(cfg)
    osv = po.Solver(ospot, prune=False, use_iso=False, exact=True)
    spot = g.Spot(cfg)
    host = g.Solver(spot, use_iso=False)
    osv.iterate(5)
    g0 = g.GpuSolver(host, engine=engine)
    g0.iterate(5)
    g0.sync_to_cpu(host)
    g0.close()
    t = spot.tree()
    child = int(spot.children()[int(t["child_start"][0])])
    na1 = int(t["nchild"][child])
    freqs = [0.4] + [0.6 / (na1 - 1)] * (na1 - 1)
    assert osv.lock_node([], 0) == host.lock_node([], "freeze") == 0
    assert osv.lock_node([0], 1, freqs=freqs) == host.lock_node([0], "range", freqs=freqs) == child
    osv.iterate(12)
    gpu = g.GpuSolver(host, engine=engine)
    gpu.iterate(12)
    gpu.sync_to_cpu(host)
    _compare(spot, osv, host, "locks/" + engine)
    eo, eg = osv.exploitability(), gpu.exploitability(host)
    assert abs(eo - eg) / 60.0 * 100 < EXPL_TOL_PCT, (eo, eg)


@pytest.mark.parametrize("algo", ["dcfr", "pcfr+"])
@pytest.mark.parametrize("name,cfg_fn,iters", [
    ("small_flop", W.small_flop_spot, 15),
    ("river_1081", W.river_spot, 10),
])
def test_fp8_arenas_match_oracle(name, cfg_fn, iters, algo):
    """FP8 E4M3 device arenas (the precision study; staged engine) against the
    oracle's FP8 arenas: the same codes in > 99.9% of entries, average
    strategies within 1e-4, exploitability within 0.01% of the pot."""
    cfg = cfg_fn()
    ospot = po.Spot(cfg)
    osv = po.Solver(ospot, fp8=True, algo=algo, prune=False, exact=True)
    osv.iterate(iters)
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", algo=algo)
    gpu = g.GpuSolver(host, device_format="fp8")
    gpu.iterate(iters)
    gpu.sync_to_cpu(host)
    for which in (0, 1):
        for p in (0, 1):
            a, b = osv.arena(which, p), host.arena(which, p)
            frac = float(np.mean(a == b))
            assert frac > 0.999, (name, algo, which, p, frac)
    so = _avg_strategies(spot, lambda p: osv.arena(1, p))
    sg = _avg_strategies(spot, lambda p: host.arena(1, p))
    worst = max(float(np.abs(so[n] - sg[n]).max()) for n in so)
    assert worst < STRAT_TOL, (name, algo, worst)
    pot = cfg["tree"]["starting_pot"]
    eo, eg = osv.exploitability(), gpu.exploitability(host)
    assert abs(eo - eg) / pot * 100 < EXPL_TOL_PCT, (eo, eg)
