"""Pins the CPU oracle to the reference's own known-answer tests and logs.

Sources (paths inside the reference project):
  evaluator.rs:304-392   known hands, 20k random deals vs best-of-21, straight_top
  cards.rs:127-215       combo bijection, canonical flops and subsets
  store.rs:221-262       i16/u16 round trips, zero / non-finite blocks
  range.rs:313-376       range parser
  convergence.rs         clairvoyance, small flop, compressed vs f32, PCFR+
  bench/*.log            bench_spot.json tree size and exploitability trajectory
"""
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from gtopen_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
L = po.lib()


def cards(s):
    out = np.zeros(16, np.uint8)
    n = L.orc_parse_cards(s.encode(), po.ptr(out), 16)
    assert n >= 0
    return out[:n]


def ev(s):
    return L.orc_evaluate7(po.ptr(cards(s)))


def test_known_hands():  # evaluator.rs:304-330
    assert ev("AsKsQsJsTs2c2d") > ev("AcAdAhAs2c2d2h")
    assert ev("As2s3s4s5s9c9d") >> 20 == 8
    assert ev("AcAdAhAsKc2d3h") > ev("AcAdAhAsQc2d3h")
    assert ev("KcKdKh2c2d2h3s") >> 20 == 6
    assert ev("KcKdKh3c3d2h2s") > ev("KcKdKh2c2d4h5s")
    assert ev("2c4c6c8cTcAdKd") > ev("3c4d5h6s7c2d2h")
    assert ev("6c5d4h3s2cKdQd") > ev("Ac5d4h3s2cKdQd")
    assert ev("AsKsQsJsTs2c3d") == ev("AsKsQsJsTs4c5d")
    assert ev("KcKdKh2c2d4h4s") > ev("KcKdKh3c3d3h9s")  # full_house_better_pair


def _ref7(c):
    cat = np.zeros(1, np.uint32)
    r = np.zeros(5, np.uint8)
    n = np.zeros(1, np.int32)
    L.orc_ref_eval7(po.ptr(c), po.ptr(cat), po.ptr(r), po.ptr(n))
    return (int(cat[0]), tuple(int(x) for x in r[: n[0]]))


def test_matches_reference_random():  # evaluator.rs:340-366
    rng = W.XorShift(0x9E3779B97F4A7C15)
    for _ in range(20000):
        deck = list(range(52))
        for i in range(14):
            j = i + rng.next() % (52 - i)
            deck[i], deck[j] = deck[j], deck[i]
        h1 = np.array(deck[0:7], np.uint8)
        h2 = np.array(deck[7:14], np.uint8)
        f1, f2 = L.orc_evaluate7(po.ptr(h1)), L.orc_evaluate7(po.ptr(h2))
        r1, r2 = _ref7(h1), _ref7(h2)
        assert f1 >> 20 == r1[0] and f2 >> 20 == r2[0]
        assert (f1 > f2) - (f1 < f2) == (r1 > r2) - (r1 < r2)


def test_straight_top_exhaustive():  # evaluator.rs:368-392
    for mask in range(1 << 13):
        exp = -1
        for top in range(12, 3, -1):  # five-card runs ending at rank >= 4; the wheel below
            need = sum(1 << (top - i) for i in range(5))
            if mask & need == need:
                exp = top
                break
        if exp < 0 and mask & ((1 << 12) | 0b1111) == ((1 << 12) | 0b1111):
            exp = 3
        assert L.orc_straight_top(mask) == exp, mask


def test_combo_index_bijection():  # cards.rs:134-146
    seen = set()
    hi, lo = po.C.c_int(), po.C.c_int()
    for c1 in range(52):
        for c2 in range(c1):
            idx = L.orc_combo_index(c1, c2)
            assert 0 <= idx < 1326 and idx not in seen
            seen.add(idx)
            L.orc_combo_from_index(idx, po.C.byref(hi), po.C.byref(lo))
            assert (hi.value, lo.value) == (c1, c2)
    assert len(seen) == 1326


def _flops(n=None):
    b = np.zeros(1755 * 6, np.uint8)
    w = np.zeros(1755, np.uint32)
    k = L.orc_canonical_flops(po.ptr(b), po.ptr(w), 1755) if n is None else \
        L.orc_canonical_flops_subset(n, po.ptr(b), po.ptr(w), 1755)
    return [bytes(b[6 * i: 6 * i + 6]).decode() for i in range(k)], w[:k]


def test_canonical_flops():  # cards.rs:183-191, 157-181
    boards, w = _flops()
    assert len(boards) == 1755 and int(w.sum()) == 22100
    for n in (1, 47, 95, 184, 500, 922, 923, 924, 1000, 1200, 1754):
        b, ww = _flops(n)
        assert len(set(b)) == len(b) and len(b) <= n and int(ww.sum()) == n
    for n in (47, 95, 184):
        b, ww = _flops(n)
        assert len(b) == n and (ww == 1).all()


def test_store_roundtrips():  # store.rs:221-262
    src = (np.sin(np.arange(1000, dtype=np.float32) * np.float32(0.7)) * 1500 - 200).astype(np.float32)
    q = np.zeros(1000, np.int16)
    sc = L.orc_encode_i16(po.ptr(src), 1000, po.ptr(q))
    back = np.zeros(1000, np.float32)
    L.orc_decode_i16(po.ptr(q), 1000, sc, po.ptr(back))
    assert np.abs(src - back).max() <= sc / 32767 * 0.5 + 1e-6
    q2 = np.zeros(1000, np.int16)
    assert L.orc_encode_i16(po.ptr(back), 1000, po.ptr(q2)) == sc and (q == q2).all()
    us = (np.abs(np.cos(np.arange(1000, dtype=np.float32) * np.float32(0.37))) * 9.5).astype(np.float32)
    qu = np.zeros(1000, np.uint16)
    sc = L.orc_encode_u16(po.ptr(us), 1000, po.ptr(qu))
    L.orc_decode_u16(po.ptr(qu), 1000, sc, po.ptr(back))
    assert np.abs(us - back).max() <= sc / 65535 * 0.5 + 1e-6
    z = np.zeros(4, np.float32)
    q = np.full(4, 7, np.int16)
    assert L.orc_encode_i16(po.ptr(z), 4, po.ptr(q)) == 0.0 and (q == 0).all()
    nf = np.array([np.nan, np.inf], np.float32)
    q = np.full(2, 7, np.int16)
    assert L.orc_encode_i16(po.ptr(nf), 2, po.ptr(q)) == 0.0 and (q == 0).all()


def _count(s):
    w = np.zeros(1326, np.float32)
    assert L.orc_parse_range(s.encode(), po.ptr(w)) == 0
    return float(w.sum()), w


def test_range_parser():  # range.rs:313-376
    for s, n in [("AA", 6), ("AKs", 4), ("AKo", 12), ("AK", 16), ("AhKh", 1), ("TT+", 30), ("ATs+", 16),
                 ("99-66", 24), ("A5s-A2s", 16), ("T9s-87s", 12), ("AA,KK,QQ", 18)]:
        assert _count(s)[0] == n, s
    _, w = _count("AA:0.5,KK")
    assert abs(w[L.orc_combo_index(48, 49)] - 0.5) < 1e-6 and abs(w[L.orc_combo_index(44, 45)] - 1.0) < 1e-6
    _, w = _count("AA:50")
    assert abs(w[L.orc_combo_index(48, 49)] - 0.5) < 1e-6
    _, w = _count("AA,AA:0.25")
    assert abs(w[L.orc_combo_index(48, 49)] - 0.25) < 1e-6
    _, w = _count("AKs:1.5")
    assert abs(w[L.orc_combo_index(48, 44)] - 0.015) < 1e-6
    for bad in ("XX", "AAs", "AKs:abc"):
        assert L.orc_parse_range(bad.encode(), po.ptr(np.zeros(1326, np.float32))) != 0


def test_bench_spot_tree_pins():  # bench/new_f32_dcfr.log line 1
    cfg = json.load(open(os.path.join(HERE, "golden", "bench_spot.json")))
    s = po.Spot(cfg)
    assert s.num_nodes == 1245971
    assert int((s.nodes()["kind"] == 0).sum()) == 500748
    assert s.nh == [257, 319]
    ds = sum(s.data_size)
    assert round(ds * 8 / 1e6, 1) == 2494.8
    assert round((ds * 4 + s.num_nodes * 16) / 1e6, 1) == 1267.3


def test_bench_spot_first_checkpoint():
    """bench/new_f32_dcfr.log: 33.7904 chips (56.317% pot) after 10 DCFR iterations."""
    cfg = json.load(open(os.path.join(HERE, "golden", "bench_spot.json")))
    s = po.Spot(cfg)
    sv = po.Solver(s, compressed=False, algo="dcfr", use_iso=True, prune=True)
    sv.iterate(10)
    e = sv.exploitability()
    assert "%.4f" % e == "33.7904"
    assert "%.3f" % (e / 60 * 100) == "56.317"


def test_bench_trajectory_golden():
    """The committed full trajectories (tests/golden/make_bench_trajectory.py) equal the
    reference's printed logs for f32 DCFR, i16 DCFR and i16 PCFR+."""
    g = json.load(open(os.path.join(HERE, "golden", "bench_trajectory.json")))
    for mode, d in g["modes"].items():
        assert len(d["oracle"]) == 10, mode
        for a, b in zip(d["oracle"], d["reference"]):
            assert "%.4f" % a == "%.4f" % b, (mode, a, b)


def test_exact_sums_reproduce_reference_logs():
    """The exact fixed-point terminal sums (the GPU engine's arithmetic) with
    the reference CPU engine's pruning reproduce the reference's printed CPU
    logs (bench/new_f32_dcfr.log, new_i16_dcfr.log) to the printed digits at
    all ten checkpoints; without pruning they stay within 0.001% of the pot
    of the f64 sums.  Recorded by tests/golden/make_noprune_trajectory.py."""
    g = json.load(open(os.path.join(HERE, "golden", "bench_trajectory_noprune.json")))
    ref = json.load(open(os.path.join(HERE, "golden", "bench_trajectory.json")))
    pot = g["pot"]
    for mode in ("f32_dcfr", "i16_dcfr"):
        for a, b in zip(g["pruned_exact"][mode], ref["modes"][mode]["reference"]):
            assert "%.4f" % a == "%.4f" % b, (mode, a, b)
        for a, b in zip(g["modes"][mode], g["modes_f64"][mode]):
            assert abs(a - b) / pot * 100 < 1e-3, (mode, a, b)


@pytest.mark.slow
def test_exact_sums_first_checkpoint_rerun():
    """Re-runs the first checkpoint of the exact-sum, pruned f32 trajectory."""
    cfg = json.load(open(os.path.join(HERE, "golden", "bench_spot.json")))
    sv = po.Solver(po.Spot(cfg), compressed=False, algo="dcfr", use_iso=True, prune=True, exact=True)
    sv.iterate(10)
    assert "%.4f" % sv.exploitability() == "33.7904"


@pytest.mark.slow
def test_bench_trajectory_rerun():
    """Re-runs the 100-iteration f32 trajectory (about 3 minutes on 8 cores)."""
    cfg = json.load(open(os.path.join(HERE, "golden", "bench_spot.json")))
    s = po.Spot(cfg)
    sv = po.Solver(s, compressed=False, algo="dcfr", use_iso=True, prune=True)
    ref = [33.7904, 9.3381, 4.8733, 3.3154, 2.3677, 1.7728, 1.3505, 1.0533, 0.8316, 0.6747]
    for k in range(10):
        sv.iterate(10)
        assert "%.4f" % sv.exploitability() == "%.4f" % ref[k]


def test_clairvoyance_converges_to_theory():  # convergence.rs:32-105
    s = po.Spot(W.clairvoyance_spot())
    sv = po.Solver(s)
    sv.iterate(3000)
    assert sv.exploitability() / 100 * 100 < 0.10
    c1, c2, _ = s.hands(0)
    names = [W.combo_str(int(a), int(b)) for a, b in zip(c1, c2)]
    nh = s.nh[0]
    sig = sv.avg_strategy(0, 2, nh)
    assert sig[nh + names.index("AcKc")] > 0.97
    assert abs(sig[nh + names.index("8h7h")] - 0.5) < 0.05


def test_small_flop_converges_and_compressed_matches():  # convergence.rs:110-136, 449-497
    cfg = W.small_flop_spot()
    s = po.Spot(cfg)
    a = po.Solver(s, compressed=False)
    b = po.Solver(s, compressed=True)
    a.iterate(200)
    b.iterate(200)
    ea, eb = a.exploitability() / 60 * 100, b.exploitability() / 60 * 100
    assert ea < 1.0 and eb < 1.0 and abs(ea - eb) < 0.1


def test_pcfr_plus_converges():  # convergence.rs:501-521
    s = po.Spot(W.small_flop_spot())
    for comp in (False, True):
        sv = po.Solver(s, compressed=comp, algo="pcfr+")
        sv.iterate(200)
        assert sv.exploitability() / 60 * 100 < 1.0


def test_fp64_oracle_agrees_with_f32_br():
    s = po.Spot(W.small_flop_spot())
    sv = po.Solver(s, prune=False)
    sv.iterate(50)
    e32, e64 = sv.exploitability(), sv.exploitability_f64()
    assert abs(e32 - e64) / 60 * 100 < 1e-3, (e32, e64)


def test_fp8_codec_matches_e4m3fn():
    """The oracle's FP8 E4M3 codec (the precision-study arenas): every code
    decodes like torch's float8_e4m3fn, in-range floats round like it
    (nearest, ties to even), and out-of-range values saturate to +-448."""
    import torch
    dec = po.fp8_decode(np.arange(256, dtype=np.uint8))
    ref = torch.arange(256, dtype=torch.uint8).view(torch.float8_e4m3fn).float().numpy()
    assert np.all((dec == ref) | (np.isnan(dec) & np.isnan(ref)))
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.standard_normal(100000).astype(np.float32) * s for s in (1e-3, 0.05, 1.0, 30.0, 200.0)])
    x = np.clip(x, -448.0, 448.0).astype(np.float32)
    # exact midpoints between neighbouring codes (ties go to the even code)
    fin = np.sort(np.unique(ref[np.isfinite(ref) & (ref >= 0)]))
    mids = ((fin[:-1].astype(np.float64) + fin[1:]) / 2).astype(np.float32)
    x = np.concatenate([x, mids, -mids])
    q = po.fp8_encode(x)
    t = torch.from_numpy(x).to(torch.float8_e4m3fn).view(torch.uint8).numpy()
    assert int((q != t).sum()) == 0
    big = np.array([448.0, 449.0, 464.0, 1e6, -500.0, np.inf, -np.inf], np.float32)
    assert list(po.fp8_encode(big)) == [0x7E, 0x7E, 0x7E, 0x7E, 0xFE, 0x7E, 0xFE]


def test_fp8_arenas_precision_study():
    """Precision study (small flop, f64 best response): FP8 E4M3 arenas with a
    per-node scale and round-to-nearest converge at first, then stall near
    3.3% of the pot -- increments below the format's 3-bit mantissa no longer
    change the stored regrets and strategy sums -- where f32 and the 16-bit
    format keep converging (0.08% and 0.11% after 300 iterations)."""
    spot = po.Spot(W.small_flop_spot())
    pot = W.small_flop_spot()["tree"]["starting_pot"]
    res = {}
    for name, kw in (("f32", {}), ("i16", {"compressed": True}), ("fp8", {"fp8": True})):
        sv = po.Solver(spot, prune=False, **kw)
        sv.iterate(10)
        first = sv.exploitability_f64() / pot * 100
        sv.iterate(290)
        res[name] = (first, sv.exploitability_f64() / pot * 100)
    assert res["f32"][1] < 0.1 and res["i16"][1] < 0.15
    assert res["fp8"][1] < res["fp8"][0] and res["fp8"][1] < 4.0
    assert res["fp8"][1] > 10 * res["f32"][1]  # the stall, as recorded


def _exact_terms_numpy(spot, p, dealt, ro, win, lose, tie):
    """Independent restatement of the exact terminal sums: every opponent
    reach value on the grid 2^-S (S = 51 - E, the vector's max < 2^E), the
    compatible weaker / stronger / all opponent mass of each hand summed by
    explicit masks in int64, each sum to f32 once, then the reference's f32
    arithmetic (game.rs:470-577)."""
    o = 1 - p
    c1m, c2m, _ = spot.hands(p)
    c1o, c2o, _ = spot.hands(o)
    mx = float(ro.max())
    S = 51 - np.frexp(mx)[1] if mx > 0 else 0
    q = np.rint(ro.astype(np.float64) * 2.0 ** S).astype(np.int64)

    def f32(x):
        return np.float32(np.int64(x)) * np.float32(2.0 ** -S)

    st_m, ix_m = spot.river(p, dealt)
    st_o, ix_o = spot.river(o, dealt)
    strength_o = np.full(len(c1o), -1, np.int64)
    strength_o[ix_o] = st_o
    fold = np.zeros(len(c1m), np.float32)
    show = np.zeros(len(c1m), np.float32)
    pos = {int(i): int(s) for s, i in zip(st_m, ix_m)}
    for i in range(len(c1m)):
        dis = (c1o != c1m[i]) & (c1o != c2m[i]) & (c2o != c1m[i]) & (c2o != c2m[i])
        same = np.nonzero((np.minimum(c1o, c2o) == min(c1m[i], c2m[i])) & (np.maximum(c1o, c2o) == max(c1m[i], c2m[i])))[0]
        q_same = int(q[same[0]]) if len(same) else 0
        same_r = np.float32(ro[same[0]]) if len(same) else np.float32(0)
        valid = np.float32(f32(int(q[dis].sum()) - q_same) + same_r)
        fold[i] = np.float32(10.0) * valid
        if i in pos:
            s = pos[i]
            ok = dis & (strength_o >= 0)
            lo = f32(int(q[ok & (strength_o < s)].sum()))
            hi = f32(int(q[ok & (strength_o > s)].sum()))
            # valid over the board's hands: total minus the two card sums (the same combo counted twice)
            on = strength_o >= 0
            has1 = (c1o == c1m[i]) | (c2o == c1m[i])
            has2 = (c1o == c2m[i]) | (c2o == c2m[i])
            vq = int(q[on].sum()) - int(q[on & has1].sum()) - int(q[on & has2].sum())
            va = np.float32(f32(vq) + same_r)
            ti = np.float32(np.float32(va - lo) - hi)
            show[i] = np.float32(np.float32(np.float32(np.float32(win) * lo) + np.float32(np.float32(lose) * hi))
                                 + np.float32(np.float32(tie) * ti))
    return fold, show


def test_exact_terminal_sums_restated():
    """The oracle's exact fold and showdown sums (the GPU engine's
    arithmetic) equal an independent numpy restatement bit for bit, on reach
    vectors of ordinary, tiny (1e-25) and mixed magnitudes; and they stay
    within a few f32 rounding steps of the reference's f64 running sums."""
    cfg = W.small_flop_spot()
    spot = po.Spot(cfg)
    rng = np.random.default_rng(11)
    dealt = [int(c) for c in rng.choice([c for c in range(52) if c not in cards(cfg["board"])], 2, replace=False)]
    c1o, c2o, _ = spot.hands(1)
    blocked = np.isin(c1o, dealt) | np.isin(c2o, dealt)
    for scale in (1.0, 1e-25, None):
        ro = rng.random(spot.nh[1]).astype(np.float32)
        ro[rng.random(spot.nh[1]) < 0.2] = 0.0
        if scale is None:
            ro *= (10.0 ** rng.integers(-30, 1, spot.nh[1])).astype(np.float32)
        else:
            ro *= np.float32(scale)
        ro[blocked] = 0.0
        win, lose, tie = 37.5, -37.5, 0.0
        fold, show = _exact_terms_numpy(spot, 0, dealt, ro, win, lose, tie)
        a = spot.fold_cfv(0, ro, 10.0, exact=True)
        b = spot.showdown_cfv(0, dealt, ro, win, lose, tie, exact=True)
        st, ix = spot.river(0, dealt)
        assert np.array_equal(a.view(np.uint32), fold.view(np.uint32)), scale
        assert np.array_equal(b[ix].view(np.uint32), show[ix].view(np.uint32)), scale
        a64 = spot.fold_cfv(0, ro, 10.0)
        b64 = spot.showdown_cfv(0, dealt, ro, win, lose, tie)
        big = max(float(np.abs(a64).max()), 1e-45)
        assert float(np.abs(a - a64).max()) <= 4 * np.finfo(np.float32).eps * big, scale
        bigs = max(float(np.abs(b64).max()), 1e-45)
        assert float(np.abs(b - b64).max()) <= 64 * np.finfo(np.float32).eps * bigs, scale
