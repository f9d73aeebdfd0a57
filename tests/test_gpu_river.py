"""River programs (engine "staged_river": one CTA walks a whole river betting
round depth first) against the staged engine's level-synchronous sweeps on the
same spots: the arithmetic is the same, so after the same iterations every arena entry, the
per-node scales (through the decoded arenas) and the exploitability are equal
bit for bit -- f32, 16-bit (round to nearest and stochastic rounding) and FP8
arenas, DCFR, CFR+ and PCFR+, with and without suit isomorphism, with a locked
river node, and on a river spot whose root is itself a river round.
"""
import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _iso_spot():
    cfg = W.small_flop_spot()
    cfg["board"] = "Qs8h3d"  # rainbow flop: suit symmetries with uniform ranges
    return cfg


SPOTS = {
    "small_flop": W.small_flop_spot,
    "iso_flop": _iso_spot,
    "river_1081": lambda: W.river_spot(seed=1),
    "turn_c2": lambda: W.turn_spot(g.evaluate7, seed=2),
}


def _pair(cfg, storage, device_format, algo, use_iso, iters, lock=None):
    out = []
    for engine in ("staged_river", "staged"):
        spot = g.Spot(cfg)
        host = g.Solver(spot, storage=storage, algo=algo, use_iso=use_iso)
        if lock is not None:
            lock(spot, host)
        gpu = g.GpuSolver(host, device_format=device_format, engine=engine)
        gpu.iterate(iters)
        e = gpu.exploitability(host)
        kinds = (0, 1, 2) if algo == "pcfr+" else (0, 1)
        arenas = {(w, p): gpu.export_arena(w, p).copy() for w in kinds for p in (0, 1)}
        out.append((gpu.info()["river_programs"], e, arenas))
        gpu.close()
    return out


@pytest.mark.parametrize("name", list(SPOTS))
@pytest.mark.parametrize("storage,device_format", [("f32", None), ("compressed", None), ("compressed", "i16sr"),
                                                   ("f32", "fp8")])
def test_river_programs_equal_level_sweeps(name, storage, device_format):
    cfg = SPOTS[name]()
    (nr, e_r, a_r), (nl, e_l, a_l) = _pair(cfg, storage, device_format, "dcfr", name == "iso_flop", 12)
    assert nr > 0 and nl == 0
    assert e_r == e_l, (name, storage, device_format, e_r, e_l)
    for key in a_r:
        diff = int(np.count_nonzero(a_r[key].view(np.uint32) != a_l[key].view(np.uint32)))
        assert diff == 0, (name, storage, device_format, key, diff)


@pytest.mark.parametrize("algo", ["cfr+", "pcfr+"])
@pytest.mark.parametrize("storage", ["f32", "compressed"])
def test_river_programs_cfrplus_pcfrplus(algo, storage):
    (nr, e_r, a_r), (nl, e_l, a_l) = _pair(W.small_flop_spot(), storage, None, algo, False, 10)
    assert nr > 0 and nl == 0 and e_r == e_l
    for key in a_r:
        assert np.array_equal(a_r[key].view(np.uint32), a_l[key].view(np.uint32)), (algo, storage, key)


def test_river_programs_with_a_locked_river_node():
    cfg = W.small_flop_spot()
    board = cfg["board"]
    turn, river = [c for c in ("2c", "3c", "4c", "5c") if c not in board][:2]
    path = [0, 0, turn, 0, 0, river, 0]  # checks through to the river, IP's node after OOP checks

    def lock(spot_, host):
        host.lock_node([0, 0, turn, 0, 0, river], "range", freqs=[0.0, 1.0])
        host.lock_node(path, "freeze")

    (nr, e_r, a_r), (nl, e_l, a_l) = _pair(cfg, "f32", None, "dcfr", False, 10, lock=lock)
    assert nr > 0 and e_r == e_l
    for key in a_r:
        assert np.array_equal(a_r[key].view(np.uint32), a_l[key].view(np.uint32)), key


def test_river_programs_best_response_and_average_sweeps():
    cfg = W.small_flop_spot()
    vals = []
    for engine in ("staged", "staged_river"):
        spot = g.Spot(cfg)
        host = g.Solver(spot, storage="compressed", algo="dcfr", use_iso=False)
        gpu = g.GpuSolver(host, engine=engine)
        gpu.iterate(8)
        vals.append([gpu.root_cfv(p, m).copy() for p in (0, 1) for m in (0, 1)])
        gpu.close()
    for a, b in zip(*vals):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
