"""Training data and training for the turn-leaf value network of a
depth-limited flop solve.

A depth-limited solve cuts the flop tree at the chance nodes that deal the
turn where betting follows; each such leaf is a turn spot (the flop plus one
turn card, the pot and remaining stack at the leaf, the players' reach as
ranges).  The network maps one such turn spot to both players' root
counterfactual values.  Training samples are turn spots of the flop being
solved, with the (pot, stack) of one of its leaves and seeded random ranges
over its hands, each solved by the plain engine (many at once on one GPU,
gtob_batch_*); the target is the solved root's counterfactual values.

Input row (LEAF_IN = 2705 values), as the device gather builds it:
  [0, 52)          one-hot of the three flop cards and the turn card
  52               pot / remaining stack
  [53, 1379)       player 0's reach over the 1326 combos / its sum
  [1379, 2705)     player 1's, the same way
Output row (LEAF_OUT = 2652): per player the combos' counterfactual values /
(pot x the opponent's reach sum); only the combos of the player's hands are
trained (mask 1).
"""
import copy

import numpy as np

from . import workloads as W

LEAF_IN = 52 + 1 + 2 * 1326
LEAF_OUT = 2 * 1326


def combo_index(c1, c2):
    hi = np.maximum(c1, c2).astype(np.int64)
    lo = np.minimum(c1, c2).astype(np.int64)
    return hi * (hi - 1) // 2 + lo


def dl_flop_spot(evaluate7, seed=5):
    """The depth-limited configuration's flop: the turn configuration's spot
    (top 50% of combos each side, weights U[0.2,1], pot 100, stack 300, bets
    {33,75,a}, raise 2.5x, 2 raises) on a seeded flop, with the donk sizes
    equal to the bet sizes so that every turn subtree is the tree of the turn
    spot with the same pot and stack."""
    rng = W.XorShift(seed)
    board = W.draw_board(rng, 3)
    r = [W.weighted_range(rng, W.top_fraction(rng, board, 0.5, evaluate7), 0.2) for _ in range(2)]
    return {"board": "".join(W.card_str(c) for c in board), "range_oop": r[0], "range_ip": r[1],
            "tree": W.tree_config(100, 300, ("33", "75", "a"), ("2.5x",), 2, donk=("33", "75", "a"))}


def leaf_row(board3, turn, pot, stack, hands, reach):
    """One input row and the reach sums: hands[q] = (c1, c2) arrays, reach[q]
    per hand (f32).  Hands holding the turn card count as zero."""
    x = np.zeros(LEAF_IN, np.float32)
    for c in list(board3) + [turn]:
        x[c] = 1.0
    x[52] = np.float32(pot) / np.float32(stack)
    mass = [0.0, 0.0]
    for q in range(2):
        c1, c2 = hands[q]
        r = np.where((c1 == turn) | (c2 == turn), 0.0, reach[q]).astype(np.float32)
        m = np.float32(r.sum(dtype=np.float32))
        mass[q] = m
        if m > 0:
            x[53 + q * 1326 + combo_index(c1, c2)] = r * (np.float32(1.0) / m)
    return x, mass


def leaf_values(y_rows, x_rows, masses, cards, pot, hands, p):
    """A leaf's values for player p from the net's output rows (one per turn
    card, in `cards` order): zero-sum correction, scale back, sum over the
    cards a hand does not hold, x 1/45 -- the device scatter's arithmetic."""
    c1, c2 = hands[p]
    cb = combo_index(c1, c2)
    acc = np.zeros(len(c1), np.float32)
    for j, c in enumerate(cards):
        x = x_rows[j]
        err = np.float32(np.dot(x[53:53 + 2 * 1326].astype(np.float64), y_rows[j].astype(np.float64)))
        v = (y_rows[j][p * 1326 + cb] - np.float32(0.5) * err) * np.float32(pot) * np.float32(masses[j][1 - p])
        acc += np.where((c1 == c) | (c2 == c), np.float32(0.0), v.astype(np.float32))
    return acc * np.float32(1.0 / 45.0)


def random_reach(rng, w, strength):
    """A seeded reach vector over a range: the weights times a random mix of
    shapes a flop strategy leaves behind (uniform thinning, a power of a
    uniform draw, strength-correlated cuts, pure folds of a random share)."""
    n = len(w)
    u = np.array([rng.uniform() for _ in range(n)])
    kind = rng.below(4)
    if kind == 0:
        f = u
    elif kind == 1:
        f = u ** (1 + rng.below(4))
    elif kind == 2:  # keep the strong (or the weak) end, softly
        t = rng.uniform()
        s = strength if rng.below(2) else 1.0 - strength
        f = 1.0 / (1.0 + np.exp(-(s - t) * 12.0)) * (0.5 + 0.5 * u)
    else:
        f = np.where(u < 0.2 + 0.6 * rng.uniform(), 0.0, 0.5 + 0.5 * u)
    return (np.asarray(w, np.float64) * f).astype(np.float32)


def turn_spot_config(board3, turn, pot, stack, hands, reach, tree, floor=1e-4):
    """The turn spot of one leaf: every hand not holding the turn card, its
    reach as its weight (at least floor x the largest, so that every hand
    gets a value)."""
    board = "".join(W.card_str(c) for c in list(board3) + [turn])
    rs = []
    for q in range(2):
        c1, c2 = hands[q]
        r = reach[q]
        top = float(r.max()) if len(r) and r.max() > 0 else 1.0
        toks = []
        for i in range(len(c1)):
            if c1[i] == turn or c2[i] == turn:
                continue
            wv = max(float(r[i]), floor * top)
            toks.append("%s:%.6f" % (W.combo_str(int(c1[i]), int(c2[i])), min(wv / top, 1.0)))
        rs.append(",".join(toks))
    t = dict(tree)
    t["starting_pot"] = float(pot)
    t["effective_stack"] = float(stack)
    return {"board": board, "range_oop": rs[0], "range_ip": rs[1], "tree": t}


def training_set(g, flop_cfg, leaf_pots, n, seed=1, max_iterations=300, target_pct=0.3, workers=16,
                 build_pool=None):
    """n turn spots of the flop (turn card, one leaf's (pot, stack), random
    ranges), solved on the GPU; returns (X, T, M, info): inputs, targets,
    masks (n x 2705 / 2652) and the solves' exploitability (% pot)."""
    spot = g.Spot(flop_cfg)
    board3 = [W.RANKS.index(flop_cfg["board"][i].upper()) * 4 + W.SUITS.index(flop_cfg["board"][i + 1])
              for i in range(0, 6, 2)]
    hands = []
    for q in range(2):
        c1, c2, w, _ = spot.hands(q)
        hands.append((c1.astype(np.int64), c2.astype(np.int64), w))
    # strength proxy per hand: its flop evaluation with two seeded runout cards
    rng = W.XorShift(seed * 7919 + 13)
    runout = [c for c in W.draw_board(rng, 52) if c not in board3][:2]
    strength = []
    for q in range(2):
        c1, c2, _ = hands[q]
        vals = np.array([g.evaluate7(list(board3) + runout + [int(a), int(b)])
                         if int(a) not in runout and int(b) not in runout else 0 for a, b in zip(c1, c2)], float)
        order = np.argsort(np.argsort(vals))
        strength.append(order / max(len(order) - 1, 1))
    cards = [c for c in range(52) if c not in board3]
    tree = flop_cfg["tree"]
    cfgs, rows_in = [], []
    for k in range(n):
        turn = cards[rng.below(len(cards))]
        pot, stack = leaf_pots[rng.below(len(leaf_pots))]
        reach = [random_reach(rng, hands[q][2], strength[q]) for q in range(2)]
        for q in range(2):  # a range that vanished: keep one hand alive
            if not (reach[q] > 0).any():
                reach[q][rng.below(len(reach[q]))] = hands[q][2].max()
        cfgs.append(turn_spot_config(board3, turn, pot, stack, [h[:2] for h in hands], reach, tree))
        rows_in.append((turn, pot, stack))
    spots = list(build_pool.map(g.Spot, cfgs)) if build_pool else [g.Spot(c) for c in cfgs]
    batch = g.Batch(spots, storage="f32", use_iso=False, device_format="f32", keep_solvers=False)
    batch.run(max_iterations=max_iterations, target_pct=target_pct, check_every=50, workers=workers)
    rows = batch.rows()
    X = np.zeros((n, LEAF_IN), np.float32)
    T = np.zeros((n, LEAF_OUT), np.float32)
    M = np.zeros((n, LEAF_OUT), np.float32)
    pcts = np.zeros(n)
    for k in range(n):
        if rows[k]["error"]:
            raise RuntimeError("turn spot %d: %s" % (k, rows[k]["error"]))
        turn, pot, stack = rows_in[k]
        sp = spots[k]
        th = []
        for q in range(2):
            c1, c2, w, _ = sp.hands(q)
            th.append((c1.astype(np.int64), c2.astype(np.int64), w.astype(np.float32)))
        x, mass = leaf_row(board3, turn, pot, stack, [t[:2] for t in th], [t[2] for t in th])
        X[k] = x
        for q in range(2):
            cfv = batch.root_cfv(k, q)
            opp = float(th[1 - q][2].sum(dtype=np.float64))
            cb = combo_index(th[q][0], th[q][1])
            T[k, q * 1326 + cb] = cfv / (pot * opp)
            M[k, q * 1326 + cb] = 1.0
        pcts[k] = rows[k]["exploit_pct"]
    return X, T, M, {"exploit_pct": pcts, "board3": board3, "cards": cards}


# ---------------------------------------------------------------- judging
def flop_action_nodes(spot):
    """(node, player, num_actions) of every flop action node."""
    t = spot.tree()
    idx = np.where((t["kind"] == 0) & (t["street"] == 0))[0]
    return [(int(n), int(t["player"][n]), int(t["nchild"][n])) for n in idx]


def pair_mass(spot):
    """sum over card-disjoint hand pairs of w0 * w1 (f64)."""
    c1a, c2a, w0, same0 = spot.hands(0)
    c1b, c2b, w1, _ = spot.hands(1)
    w0 = w0.astype(np.float64)
    w1 = w1.astype(np.float64)
    s = np.zeros(52)
    np.add.at(s, c1b.astype(np.int64), w1)
    np.add.at(s, c2b.astype(np.int64), w1)
    ok = same0 != 0xFFFFFFFF
    same_w = np.where(ok, w1[np.where(ok, same0, 0).astype(np.int64)], 0.0)
    valid = w1.sum() - s[c1a.astype(np.int64)] - s[c2a.astype(np.int64)] + same_w
    return float(np.dot(w0, valid))


def root_value(gpu, spot, p, pm):
    """Player p's value at the root under the average strategies, chips per
    unit of pair mass."""
    cfv = gpu.root_cfv(p, mode=1).astype(np.float64)
    w = spot.hands(p)[2].astype(np.float64)
    return float(np.dot(w, cfv)) / pm


def dl_flop_strategies(g, gpu, spot):
    """{node: average strategy (num_actions x hands)} of a solver's flop nodes."""
    return {n: g.node_strategy(gpu, n, na, pl) for n, pl, na in flop_action_nodes(spot)}


class FullTreeCheck:
    """An exact check of a flop strategy on the full tree: player p's flop
    nodes locked to it, the rest of the tree solved (both players free
    everywhere else), p's game value compared with the unlocked solve's.
    The loss (% pot) is what committing to that flop strategy costs p against
    the best continuation; each solve's exploitability bounds its noise."""

    def __init__(self, g, cfg, iterations=400, device_format="i16"):
        self.g = g
        self.cfg = cfg
        self.spot = g.Spot(cfg)
        self.host = g.Solver(self.spot, storage="compressed", use_iso=False)
        self.pot = cfg["tree"]["starting_pot"]
        self.pm = pair_mass(self.spot)
        self.iterations = iterations
        self.device_format = device_format
        self.full, self.full_exploit = self._solve({})

    def _solve(self, locks):
        self.host.clear_locks()
        for n, sigma in locks.items():
            self.host.set_lock(n, sigma)
        gpu = self.g.GpuSolver(self.host, device_format=self.device_format)
        gpu.iterate(self.iterations)
        v = [root_value(gpu, self.spot, p, self.pm) for p in (0, 1)]
        e = gpu.exploitability(self.host) / self.pot * 100
        if not locks:  # the unlocked full solve: its flop strategies are the fallback's answer
            self.full_strategies = dl_flop_strategies(self.g, gpu, self.spot)
        gpu.close()
        return v, e

    def loss(self, strategies):
        """(loss of player 0, loss of player 1, exploitability of each locked
        solve), % pot."""
        out, ex = [], []
        players = {n: pl for n, pl, _ in flop_action_nodes(self.spot)}
        for p in (0, 1):
            v, e = self._solve({n: s for n, s in strategies.items() if players[n] == p})
            out.append((self.full[p] - v[p]) / self.pot * 100)
            ex.append(e)
        self.host.clear_locks()
        return out[0], out[1], ex


# Config 5's rule: the depth-limited answer stands when committing to its flop
# strategies costs the two players together at most this share of the pot on
# the full tree; otherwise the full solve answers.
FALLBACK_PCT = 0.5


def depth_limited_or_full(g, cfg, net, check, dl_iterations=400, threshold_pct=FALLBACK_PCT, device_format="f32"):
    """A depth-limited flop solve (turn leaves from `net`) with the full solve
    as its judge and fallback: the flop strategies of the depth-limited
    solve, their loss on the full tree (check: a FullTreeCheck of the same
    config), and -- when the two losses add up to more than threshold_pct of
    the pot -- the full solve's flop strategies as the answer instead.
    Returns {"path": "depth-limited" or "full", "strategies", "loss_pct"
    (both players' losses of the depth-limited strategies), "dl_s",
    "dl_exploit_pct_cut_game", "locked_solve_exploit_pct"}."""
    import time
    spot = check.spot
    host = g.Solver(spot, storage="compressed", use_iso=False)
    dl = g.dl_gpu_solver(host, net, device_format=device_format)
    t = time.perf_counter()
    dl.iterate(dl_iterations)
    dl.synchronize()
    dl_s = time.perf_counter() - t
    e_cut = dl.exploitability(host) / cfg["tree"]["starting_pot"] * 100
    strat = dl_flop_strategies(g, dl, spot)
    kern = dl.info()["iteration_kernels"]
    dl.close()
    l0, l1, ex = check.loss(strat)
    full = l0 + l1 > threshold_pct
    return {"path": "full" if full else "depth-limited",
            "strategies": check.full_strategies if full else strat,
            "loss_pct": [l0, l1], "loss_sum_pct": l0 + l1, "threshold_pct": threshold_pct,
            "dl_iterations": dl_iterations, "dl_s": dl_s, "dl_exploit_pct_cut_game": e_cut,
            "locked_solve_exploit_pct": ex, "dl_iteration_kernels": kern}


def checkdown_config(cfg):
    """The same flop with no betting on the turn and river: both players check
    them down, so every turn and river chance node leads to showdowns only --
    the non-learned leaf (showdown equity of the ranges reaching it)."""
    c = copy.deepcopy(cfg)
    for side in ("oop", "ip"):
        for st in c["tree"][side][1:]:
            st["bet"], st["raise"], st["donk"] = [], [], []
    return c


def flop_paths(spot):
    """{action path from the root (child indices): node} of the flop action nodes."""
    t = spot.tree()
    ch = spot.children()
    out, stack = {}, [(0, ())]
    while stack:
        n, key = stack.pop()
        if t["kind"][n] != 0 or t["street"][n] != 0:
            continue
        out[key] = n
        for k in range(int(t["nchild"][n])):
            stack.append((int(ch[int(t["child_start"][n]) + k]), key + (k,)))
    return out


def checkdown_flop_strategies(g, cfg, iterations=400, device_format="f32"):
    """The flop strategies of the checked-down tree (checkdown_config) solved
    in full, keyed by the nodes of `cfg`'s own tree (the flop betting is the
    same in both)."""
    spot = g.Spot(checkdown_config(cfg))
    host = g.Solver(spot, storage="compressed", use_iso=False)
    gpu = g.GpuSolver(host, device_format=device_format)
    gpu.iterate(iterations)
    strat = dl_flop_strategies(g, gpu, spot)
    gpu.close()
    mine = flop_paths(spot)
    full = flop_paths(g.Spot(cfg))
    if set(mine) != set(full):
        raise ValueError("the checked-down tree's flop differs from the full tree's")
    return {full[k]: strat[mine[k]] for k in full}
