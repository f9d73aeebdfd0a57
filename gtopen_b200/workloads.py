"""Seeded synthetic spots with the shapes of the benchmark configurations.

No public dataset is involved: boards, ranges and weights are drawn from a
xorshift64 generator (the PRNG the reference's evaluator tests use,
crates/solver/src/evaluator.rs:292-302), seeded per configuration:
  river  -- 5-card board, both ranges = every non-blocked combo, weights U(0,1]
  turn   -- 4-card board, each range the top 50% of combos by a seeded
            strength score, weights U[0.2,1], sizes {33,75,a}/{2.5x}, 2 raises
  flop   -- 3-card board, OOP top 40% / IP top 55%, weights U[0.3,1], pot 55,
            stack 975, sizes {33,75,a}, raises {2.5x,a}, 3 raises
  flop report -- 184 suit-isomorphism classes of flops drawn without
            replacement, each with the turn config's ranges (top 50% of the
            flop's 1176 combos, weights U[0.2,1]), pot 100, stack 300, raise
            2.5x, 2 raises and 1-3 bet sizes from {33,50,75,125,a}, redrawn
            until the largest tree is at most 8x the smallest
The strength score of a combo is its 7-card strength percentile on the board
completed by seeded runout cards, plus 0.25 * U, so ranges are strength-shaped.
"""
import numpy as np

RANKS = "23456789TJQKA"
SUITS = "cdhs"
MASK64 = (1 << 64) - 1


class XorShift:
    def __init__(self, seed):
        self.s = seed & MASK64 or 0x9E3779B97F4A7C15

    def next(self):
        x = self.s
        x ^= (x << 13) & MASK64
        x ^= x >> 7
        x ^= (x << 17) & MASK64
        self.s = x
        return x

    def uniform(self):  # [0, 1)
        return (self.next() >> 11) / float(1 << 53)

    def below(self, n):
        return self.next() % n


def card_str(c):
    return RANKS[c >> 2] + SUITS[c & 3]


def combo_str(hi, lo):
    return card_str(hi) + card_str(lo)


def draw_board(rng, n):
    deck = list(range(52))
    for i in range(n):
        j = i + rng.below(52 - i)
        deck[i], deck[j] = deck[j], deck[i]
    return deck[:n]


def sizes(*toks):
    out = []
    for t in toks:
        if t == "a":
            out.append("AllIn")
        elif t.endswith("x"):
            out.append({"PrevMult": float(t[:-1])})
        else:
            out.append({"PotPct": float(t)})
    return out


def tree_config(pot, stack, bet, raise_, max_raises, donk=()):
    street = {"bet": sizes(*bet), "raise": sizes(*raise_), "donk": sizes(*donk)}
    return {"starting_pot": float(pot), "effective_stack": float(stack), "rake_pct": 0.0, "rake_cap": 0.0,
            "oop": [dict(street) for _ in range(3)], "ip": [dict(street) for _ in range(3)],
            "allin_threshold": 0.85, "add_allin": False, "max_raises": int(max_raises)}


def live_combos(board):
    bm = set(board)
    return [(hi, lo) for hi in range(52) for lo in range(hi) if hi not in bm and lo not in bm]


def strength_scores(rng, board, combos, evaluate7):
    """Percentile of each combo's 7-card strength on the board completed by
    seeded runout cards (the first candidates not held by the combo), + 0.25*U."""
    need = 5 - len(board)
    cand = [c for c in draw_board(rng, 52) if c not in board]
    vals = []
    for hi, lo in combos:
        run = [c for c in cand if c != hi and c != lo][:need]
        vals.append(evaluate7(np.array(board + run + [hi, lo], np.uint8)))
    order = np.argsort(np.array(vals, np.int64), kind="stable")
    pct = np.empty(len(combos))
    pct[order] = np.arange(len(combos)) / max(len(combos) - 1, 1)
    return [pct[i] + 0.25 * rng.uniform() for i in range(len(combos))]


def weighted_range(rng, combos, lo_w):
    toks = []
    for hi, lo in combos:
        w = lo_w + (1.0 - lo_w) * rng.uniform()
        if w <= 0.0:
            w = 1e-6
        toks.append("%s:%.6f" % (combo_str(hi, lo), w))
    return ",".join(toks)


def top_fraction(rng, board, frac, evaluate7):
    combos = live_combos(board)
    sc = strength_scores(rng, board, combos, evaluate7)
    k = int(round(frac * len(combos)))
    idx = sorted(range(len(combos)), key=lambda i: -sc[i])[:k]
    return [combos[i] for i in sorted(idx)]


def river_spot(seed=1):
    """River HU solve: all 1081 combos each side, weights U(0,1], pot 100, stack 400."""
    rng = XorShift(seed)
    board = draw_board(rng, 5)
    combos = live_combos(board)
    r0 = weighted_range(rng, combos, 0.0)
    r1 = weighted_range(rng, combos, 0.0)
    return {"board": "".join(card_str(c) for c in board), "range_oop": r0, "range_ip": r1,
            "tree": tree_config(100, 400, ("33", "75", "a"), ("2.5x",), 1)}


def turn_spot(evaluate7, seed=2):
    """Turn+river precision-study spot: top 50% each side, weights U[0.2,1], pot 100, stack 300."""
    rng = XorShift(seed)
    board = draw_board(rng, 4)
    r = [weighted_range(rng, top_fraction(rng, board, 0.5, evaluate7), 0.2) for _ in range(2)]
    return {"board": "".join(card_str(c) for c in board), "range_oop": r[0], "range_ip": r[1],
            "tree": tree_config(100, 300, ("33", "75", "a"), ("2.5x",), 2)}


def flop_spot(evaluate7, seed=3, board=None, bet=("33", "75", "a"), raise_=("2.5x", "a"), max_raises=3,
              pot=55, stack=975, frac=(0.40, 0.55), lo_w=0.3):
    """Flop single-raised-pot shape: OOP top 40% / IP top 55%, weights U[0.3,1], pot 55, stack 975."""
    rng = XorShift(seed)
    b = draw_board(rng, 3) if board is None else board
    r = [weighted_range(rng, top_fraction(rng, b, f, evaluate7), lo_w) for f in frac]
    return {"board": "".join(card_str(c) for c in b), "range_oop": r[0], "range_ip": r[1],
            "tree": tree_config(pot, stack, bet, raise_, max_raises)}


def small_flop_spot():
    """The reference's own small flop fixture (tests/convergence.rs:431-444)."""
    st = {"bet": sizes("50"), "raise": sizes("60"), "donk": []}
    st2 = {"bet": sizes("50"), "raise": [], "donk": []}
    return {"board": "Th9h2c", "range_oop": "QQ,JJ,TT,99,AhKh,AsKs,87s", "range_ip": "AA,KK,AQs,JTs,T9s",
            "tree": {"starting_pot": 60.0, "effective_stack": 200.0, "rake_pct": 0.0, "rake_cap": 0.0,
                     "oop": [st, st2, st2], "ip": [st, st2, st2], "allin_threshold": 0.85, "add_allin": False,
                     "max_raises": 10}}


def clairvoyance_spot():
    """The reference's clairvoyance fixture (tests/convergence.rs:32-48)."""
    empty = {"bet": [], "raise": [], "donk": []}
    return {"board": "QcJc9c3d2d", "range_oop": "AcKc,8h7h", "range_ip": "QdQh",
            "tree": {"starting_pot": 100.0, "effective_stack": 100.0, "rake_pct": 0.0, "rake_cap": 0.0,
                     "oop": [empty, empty, {"bet": sizes("100"), "raise": [], "donk": []}],
                     "ip": [empty, empty, empty], "allin_threshold": 0.85, "add_allin": False, "max_raises": 10}}


def iso_spot():
    """The reference's two-tone suit-isomorphism fixture (tests/convergence.rs:342-357)."""
    st = {"bet": sizes("50"), "raise": [], "donk": []}
    return {"board": "KsQs2d", "range_oop": "TT,99,88,77,AKs,AQs,AJs,JTs,T9s,87s,AKo,KQo",
            "range_ip": "QQ,JJ,TT,AKs,KQs,QJs,T9s,98s,AQo",
            "tree": {"starting_pot": 60.0, "effective_stack": 200.0, "rake_pct": 0.0, "rake_cap": 0.0,
                     "oop": [st, st, st], "ip": [st, st, st], "allin_threshold": 0.85, "add_allin": False,
                     "max_raises": 10}}


def canonical_flops():
    """One flop per suit-isomorphism class (1755 classes over the 22,100
    flops, cards.rs:183-191): the class's smallest sorted card triple under
    the 24 suit permutations, with the class's flop count."""
    import itertools
    perms = list(itertools.permutations(range(4)))
    seen = {}
    for flop in itertools.combinations(range(52), 3):
        key = min(tuple(sorted((c & ~3) | pm[c & 3] for c in flop)) for pm in perms)
        seen[key] = seen.get(key, 0) + 1
    return sorted(seen.items())


def flop_report_spots(evaluate7, build_many, n=184, seed=4, max_ratio=8.0):
    """Spots of the flop report: n canonical flops sampled without
    replacement (xorshift seed), per flop the turn config's range shape and a
    bet set of 1-3 sizes from {33,50,75,125,a}; while the largest tree
    exceeds max_ratio x the smallest, the bet set of whichever extreme lies
    farther from the median is redrawn.
    build_many(list of configs) -> list of built spots (with num_nodes), so the
    caller can build them in parallel.  Returns (configs, spots)."""
    rng = XorShift(seed)
    classes = [k for k, _ in canonical_flops()]
    for i in range(len(classes) - 1, 0, -1):
        j = rng.below(i + 1)
        classes[i], classes[j] = classes[j], classes[i]
    menu = ("33", "50", "75", "125", "a")

    def bet_set():
        k = 1 + rng.below(3)
        pick = sorted({menu[rng.below(len(menu))] for _ in range(k)}, key=menu.index)
        return tuple(pick)

    cfgs = []
    for f in classes[:n]:
        board = list(f)
        r = [weighted_range(rng, top_fraction(rng, board, 0.5, evaluate7), 0.2) for _ in range(2)]
        cfgs.append({"board": "".join(card_str(c) for c in board), "range_oop": r[0], "range_ip": r[1],
                     "tree": tree_config(100, 300, bet_set(), ("2.5x",), 2)})
    spots = list(build_many(cfgs))
    for _ in range(10 * n):
        sizes_ = np.array([sp.num_nodes for sp in spots], np.float64)
        if sizes_.max() <= max_ratio * sizes_.min():
            break
        med = float(np.median(sizes_))
        # redraw the extreme farther from the median (in ratio)
        i = int(np.argmax(sizes_)) if sizes_.max() / med >= med / sizes_.min() else int(np.argmin(sizes_))
        cfgs[i]["tree"] = tree_config(100, 300, bet_set(), ("2.5x",), 2)
        spots[i] = build_many([cfgs[i]])[0]
    return cfgs, spots
