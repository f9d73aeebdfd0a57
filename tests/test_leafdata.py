"""Host side of the depth-limited configuration (no GPU): the leaf input
rows, the zero-sum correction of the scatter's host mirror, and the claim
the training data rests on -- below every betting turn leaf of the flop tree
lies exactly the tree of the turn spot with that leaf's pot and stack."""
import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import leafdata as LD
from gtopen_b200 import workloads as W


def _board3(cfg):
    b = cfg["board"]
    return [W.RANKS.index(b[i].upper()) * 4 + W.SUITS.index(b[i + 1]) for i in range(0, 6, 2)]


def _subtree_size(t, ch, root, dealt):
    """Nodes below root that a solve can reach: the flop tree builds every
    chance node over the flop's board, so a river chance node below a turn
    card still has a child for that card, which the solver skips as dealt."""
    n, stack = 0, [root]
    while stack:
        v = stack.pop()
        n += 1
        s, k = int(t["child_start"][v]), int(t["nchild"][v])
        chance = k == 52
        stack.extend(int(c) for i, c in enumerate(ch[s:s + k]) if c != 0xFFFFFFFF and not (chance and i == dealt))
    return n


def test_turn_subtrees_are_turn_spots():
    cfg = LD.dl_flop_spot(g.evaluate7)
    spot = g.Spot(cfg)
    t, ch = spot.tree(), spot.children()
    board3 = _board3(cfg)
    hands = [spot.hands(q) for q in range(2)]
    half = cfg["tree"]["starting_pot"] / 2
    leaves = 0
    for n in np.where((t["nchild"] == 52) & (t["street"] == 1))[0]:
        kids = [int(c) for c in ch[t["child_start"][n]:t["child_start"][n] + 52]]
        turn = next(c for c in range(52) if kids[c] != 0xFFFFFFFF)
        if t["kind"][kids[turn]] != 0:  # an all-in runout, kept exact
            continue
        leaves += 1
        pot = t["put0"][n] + t["put1"][n]
        stack = cfg["tree"]["effective_stack"] - (t["put0"][n] - half)
        reach = [h[2] for h in hands]
        tc = LD.turn_spot_config(board3, turn, pot, stack, [(h[0], h[1]) for h in hands], reach, cfg["tree"])
        turn_spot = g.Spot(tc)
        assert turn_spot.num_nodes == _subtree_size(t, ch, kids[turn], turn), (int(n), turn)
    assert leaves == 11


def test_leaf_row_layout():
    board3 = [0, 5, 10]
    c1 = np.array([20, 30, 40], np.int64)
    c2 = np.array([12, 13, 14], np.int64)
    reach = [np.array([1.0, 2.0, 3.0], np.float32), np.array([0.5, 0.0, 0.5], np.float32)]
    x, mass = LD.leaf_row(board3, 30, 100.0, 300.0, [(c1, c2), (c1, c2)], reach)
    assert x.shape == (LD.LEAF_IN,)
    assert sorted(np.nonzero(x[:52])[0].tolist()) == [0, 5, 10, 30]
    assert abs(x[52] - 100.0 / 300.0) < 1e-7
    assert mass[0] == np.float32(4.0) and mass[1] == np.float32(1.0)  # the hand holding the turn card drops
    r0 = x[53:53 + 1326]
    assert abs(r0.sum() - 1.0) < 1e-6 and r0[LD.combo_index(30, 13)] == 0.0
    assert abs(r0[LD.combo_index(20, 12)] - 0.25) < 1e-7


def test_leaf_values_zero_sum():
    """After the correction the corrected outputs satisfy sum r0 y0 + sum r1 y1
    = 0 per row, so the scaled leaf values are zero-sum: sum over both
    players of reach x value is 0 for any network output."""
    rng = np.random.default_rng(2)
    board3 = [0, 5, 10]
    pairs = [(a, b) for a in range(52) for b in range(a) if a not in board3 and b not in board3]
    sel = rng.choice(len(pairs), 300, replace=False)
    c1 = np.array([pairs[i][0] for i in sel], np.int64)
    c2 = np.array([pairs[i][1] for i in sel], np.int64)
    hands = [(c1, c2), (c1, c2)]
    cards = [c for c in range(52) if c not in board3][:5]
    reach = [rng.random(300).astype(np.float32), rng.random(300).astype(np.float32)]
    rows = [LD.leaf_row(board3, c, 100.0, 300.0, hands, reach) for c in cards]
    X = np.stack([r[0] for r in rows])
    masses = [r[1] for r in rows]
    Y = rng.normal(0, 1, (len(cards), LD.LEAF_OUT)).astype(np.float32)
    total = 0.0
    scale = 0.0
    for j, c in enumerate(cards):  # one card at a time: the chance node's children
        v = [LD.leaf_values(Y[j:j + 1], X[j:j + 1], masses[j:j + 1], [c], 100.0, hands, p) for p in (0, 1)]
        blocked = (c1 == c) | (c2 == c)
        for p in (0, 1):
            r = np.where(blocked, 0.0, reach[p]).astype(np.float64)
            total += float(np.dot(r, v[p]))
            scale += float(np.dot(r, np.abs(v[p])))
    assert abs(total) <= 1e-5 * scale


def test_dl_plan_cut():
    """The depth-limited plan visits the flop's betting, its 11 betting turn
    leaves (not below them) and the 4 all-in runouts in full."""
    cfg = LD.dl_flop_spot(g.evaluate7)
    spot = g.Spot(cfg)
    t, ch = spot.tree(), spot.children()
    nodes, pots, stacks, vis = g.dl_plan(spot)
    assert len(nodes) == 11
    assert sorted(set(np.round(pots, 1))) == [100.0, 166.0, 250.0, 265.0, 475.0, 512.5]
    half = cfg["tree"]["starting_pot"] / 2
    for n, p_, s_ in zip(nodes, pots, stacks):
        assert t["nchild"][n] == 52 and t["street"][n] == 1
        assert abs(p_ - (t["put0"][n] + t["put1"][n])) < 1e-3
        assert abs(s_ - (cfg["tree"]["effective_stack"] - (t["put0"][n] - half))) < 1e-3
        kids = ch[t["child_start"][n]:t["child_start"][n] + 52]
        assert not any(vis[int(c)] for c in kids if c != 0xFFFFFFFF)  # nothing below a leaf
    v = vis.astype(bool)
    # every visited action node bets on the flop; later-street nodes are runout
    # chance nodes and showdowns below all-ins
    assert np.all(t["street"][v & (t["kind"] == 0)] == 0)
    assert np.any(v & (t["kind"] == 1) & (t["street"] == 2))  # runouts deal the river too
    with pytest.raises(g.GtobError):
        g.dl_plan(g.Spot(W.turn_spot(g.evaluate7)))  # a turn spot has no turn leaves to cut


def test_checkdown_tree_keeps_the_flop():
    """The non-learned baseline's tree: the same flop betting (every flop
    action node found by the same action path, with the same actor and
    action count), and on the turn and river nothing but checks."""
    cfg = LD.dl_flop_spot(g.evaluate7)
    full, down = g.Spot(cfg), g.Spot(LD.checkdown_config(cfg))
    pf, pd = LD.flop_paths(full), LD.flop_paths(down)
    assert set(pf) == set(pd) and len(pf) > 10
    tf, td = full.tree(), down.tree()
    for k in pf:
        assert tf["player"][pf[k]] == td["player"][pd[k]] and tf["nchild"][pf[k]] == td["nchild"][pd[k]], k
    later = (td["kind"] == 0) & (td["street"] > 0)
    assert later.any() and np.all(td["nchild"][later] == 1)
    assert down.num_nodes < full.num_nodes // 10


def test_depth_limited_or_full_applies_the_threshold():
    """Config 5's rule with stand-ins for the engine (no GPU): the depth-limited
    answer stands at or below 0.5% of the pot summed over both players, and
    above it the full solve's flop strategies answer."""
    class FakeGpu:
        def iterate(self, n):
            pass

        def synchronize(self):
            pass

        def exploitability(self, host):
            return 0.1

        def info(self):
            return {"iteration_kernels": 60}

        def close(self):
            pass

    class FakeG:
        def Solver(self, *a, **k):
            return object()

        def dl_gpu_solver(self, *a, **k):
            return FakeGpu()

        def node_strategy(self, gpu, n, na, pl):
            return np.full((na, 3), 1.0 / na, np.float32)

    class FakeCheck:
        def __init__(self, losses):
            self.spot = g.Spot(LD.dl_flop_spot(g.evaluate7))
            self.losses = losses
            self.full_strategies = {"full": True}

        def loss(self, strat):
            return self.losses[0], self.losses[1], [0.05, 0.05]

    cfg = {"tree": {"starting_pot": 100.0}}
    for losses, path in (((0.2, 0.3), "depth-limited"), ((0.3, 0.25), "full"), ((4.7, 3.5), "full")):
        chk = FakeCheck(losses)
        r = LD.depth_limited_or_full(FakeG(), cfg, None, chk, dl_iterations=10)
        assert r["path"] == path, (losses, r["path"])
        assert r["loss_sum_pct"] == pytest.approx(sum(losses))
        if path == "full":
            assert r["strategies"] is chk.full_strategies
        else:
            assert r["strategies"] is not chk.full_strategies and len(r["strategies"]) > 10
