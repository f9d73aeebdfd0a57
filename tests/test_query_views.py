"""node_view's structure on the host (gtob_solver_path_view, no GPU) against
a restatement of the reference's rules over the same tree: the action labels
(tree.rs:139-169 Action::label with trim_num and Rust's rounding), the
action views and all-in detection (query.rs:353-394), the history bar
(query.rs:396-461), the node type, board, pot, puts, available cards and
the lock flag on the orbit representative (query.rs:490-640)."""
import math
import random

import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W

KINDS = ["action", "chance", "terminal_fold", "terminal_showdown"]
ACT = {0: "fold", 1: "check", 2: "call", 3: "bet", 4: "raise"}
SENTINEL = 0xFFFFFFFF


def _rust_round(x):  # f64::round: half away from zero
    return math.copysign(math.floor(abs(x) + 0.5), x)


def _trim_num(x):
    if abs(x - _rust_round(x)) < 1e-6:
        return str(int(_rust_round(x)))
    return "%.2f" % x


class Ref:
    """The reference's view rules over the spot's tree arrays."""

    def __init__(self, spot, cfg):
        self.t = spot.tree()
        self.ch = spot.children()
        self.ak, self.aa = spot.actions()
        self.stack = cfg["tree"]["effective_stack"]
        self.pot0 = cfg["tree"]["starting_pot"]
        b = cfg["board"]
        self.board = [b[i:i + 2] for i in range(0, len(b), 2)]

    def child(self, n, k):
        return int(self.ch[int(self.t["child_start"][n]) + k])

    def put(self, n, p):
        return float(self.t["put0" if p == 0 else "put1"][n])

    def actions(self, n):
        t = self.t
        if t["kind"][n] != 0:
            return []
        pot = self.put(n, 0) + self.put(n, 1)
        me = int(t["player"][n])
        out = []
        for a in range(int(t["nchild"][n])):
            k, amt = int(self.ak[int(t["action_start"][n]) + a]), float(self.aa[int(t["action_start"][n]) + a])
            all_in = False
            if k in (3, 4):
                c = self.child(n, a)
                all_in = abs(self.stack - (self.put(c, me) - self.pot0 / 2)) < 1e-6
            if k == 0:
                lab = "Fold"
            elif k == 1:
                lab = "Check"
            elif k == 2:
                lab = "Call"
            elif k == 3:
                lab = ("All-in " + _trim_num(amt)) if all_in else "Bet %s (%d%%)" % (_trim_num(amt),
                                                                                      int(_rust_round(amt / pot * 100)))
            else:
                lab = ("All-in " + _trim_num(amt)) if all_in else "Raise " + _trim_num(amt)
            out.append({"label": lab, "kind": ACT[k], "amount": amt if k in (2, 3, 4) else 0.0})
        return out

    def view(self, path):
        t = self.t
        n, dealt, hist = 0, [], []
        for s in path:
            pot = self.put(n, 0) + self.put(n, 1)
            if isinstance(s, int):
                p = int(t["player"][n])
                hist.append({"kind": "action", "player": p, "stack": self.stack - (self.put(n, p) - self.pot0 / 2),
                             "pot": pot, "street": int(t["street"][n]), "actions": self.actions(n), "chosen": s,
                             "card": None})
                n = self.child(n, s)
            else:
                c = "23456789TJQKA".index(s[0]) * 4 + "cdhs".index(s[1])
                hist.append({"kind": "card", "player": None, "stack": 0.0, "pot": pot, "street": int(t["street"][n]),
                             "actions": [], "chosen": None, "card": s})
                dealt.append(s)
                n = self.child(n, c)
        act = t["kind"][n] == 0
        p = int(t["player"][n])
        hist.append({"kind": "action" if act else ("card" if t["kind"][n] == 1 else "terminal"),
                     "player": p if act else None,
                     "stack": self.stack - (self.put(n, p) - self.pot0 / 2) if act else 0.0,
                     "pot": self.put(n, 0) + self.put(n, 1), "street": int(t["street"][n]),
                     "actions": self.actions(n), "chosen": None, "card": None})
        avail = None
        if t["kind"][n] == 1:
            avail = [g.card_string(c) for c in range(52)
                     if self.child(n, c) != SENTINEL and g.card_string(c) not in dealt]
        return {"node": n, "node_type": KINDS[int(t["kind"][n])], "street": int(t["street"][n]),
                "board": self.board + dealt, "pot": self.put(n, 0) + self.put(n, 1),
                "put": [self.put(n, 0), self.put(n, 1)], "player": p if act else None, "actions": self.actions(n),
                "available_cards": avail, "history": hist}


def _random_paths(ref, rng, n):
    t = ref.t
    out = []
    for _ in range(n):
        path, node, dealt = [], 0, set()
        for _ in range(rng.randrange(0, 12)):
            k = int(t["kind"][node])
            if k == 0:
                a = rng.randrange(int(t["nchild"][node]))
                path.append(a)
                node = ref.child(node, a)
            elif k == 1:
                cards = [c for c in range(52) if ref.child(node, c) != SENTINEL and c not in dealt]
                c = rng.choice(cards)
                dealt.add(c)
                path.append(g.card_string(c))
                node = ref.child(node, c)
            else:
                break
        out.append(path)
    return out


@pytest.mark.parametrize("cfg_fn", [W.small_flop_spot, W.iso_spot, lambda: W.river_spot(seed=1),
                                    lambda: W.flop_spot(g.evaluate7, seed=3, bet=("33", "75", "a"),
                                                        raise_=("2.5x", "a"), max_raises=2, stack=120)])
def test_path_view_matches_the_reference_rules(cfg_fn):
    cfg = cfg_fn()
    spot = g.Spot(cfg)
    sv = g.Solver(spot, use_iso=True)
    ref = Ref(spot, cfg)
    rng = random.Random(11)
    paths = [[]] + _random_paths(ref, rng, 60)
    kinds = set()
    for path in paths:
        got = sv.path_view(path)
        want = ref.view(path)
        assert got.pop("locked") is False
        assert got == want, (path, got, want)
        kinds.add(got["node_type"])
    assert "action" in kinds and len(kinds) >= 3
    labels = {a["label"].split()[0] for p in paths for a in sv.path_view(p)["actions"]}
    assert {"Check", "Bet", "Call", "Fold"} <= labels


def test_path_view_lock_flag_follows_the_representative():
    """A lock made through one card of a suit orbit shows on its isomorphic
    twin (query.rs:627-633: the lock lives on the representative's node)."""
    cfg = W.iso_spot()
    spot = g.Spot(cfg)
    sv = g.Solver(spot, use_iso=True)
    perms = spot.suit_perms()
    assert spot.num_suit_perms >= 2, perms
    ref = Ref(spot, cfg)
    # the first chance node after check-check, and a card with an isomorphic twin
    path = [0, 0]
    node = ref.child(ref.child(0, 0), 0)
    assert ref.t["kind"][node] == 1
    cards = [c for c in range(52) if ref.child(node, c) != SENTINEL]
    board_suits = {"cdhs".index(ch) for ch in cfg["board"][1::2]}
    free = [s for s in range(4) if s not in board_suits]
    twins = [(c, (c & ~3) | free[1]) for c in cards if (c & 3) == free[0]]
    c, d = twins[0]
    assert d in cards
    sv.lock_node(path + [g.card_string(c)], "freeze")
    assert sv.path_view(path + [g.card_string(c)])["locked"]
    assert sv.path_view(path + [g.card_string(d)])["locked"]
    assert not sv.path_view(path)["locked"]


def test_path_view_rejects_bad_steps():
    spot = g.Spot(W.small_flop_spot())
    sv = g.Solver(spot)
    with pytest.raises(g.GtobError):
        sv.path_view([99])
    with pytest.raises(g.GtobError):
        sv.path_view(["As"])  # a card at an action node
    assert np.isfinite(sv.path_view([0])["pot"])


def test_node_view_composes_host_structure_and_device_numbers():
    """GpuSolver.node_view's assembly (no GPU: the device numbers are stood
    in by fixed arrays): the reference's NodeView fields, combo strings as
    cards.rs prints them, NaN -> None, strategy and evs for the actor only."""
    cfg = W.small_flop_spot()
    spot = g.Spot(cfg)
    sv = g.Solver(spot)
    path = [1]
    hv = sv.path_view(path)
    na, p = len(hv["actions"]), hv["player"]
    nh = spot.nh

    def fake_values(path_, solver=None):
        ev = [np.linspace(1, 2, nh[q]).astype(np.float32) for q in (0, 1)]
        ev[p][0] = np.nan
        return {"node": hv["node"], "kind": 0, "player": p,
                "reach": [np.full(nh[q], 0.5, np.float32) for q in (0, 1)],
                "valid": [np.full(nh[q], 2.0, np.float32) for q in (0, 1)],
                "eq": [np.full(nh[q], np.nan if q else 0.25, np.float32) for q in (0, 1)], "ev": ev,
                "strategy": np.full((na, nh[p]), 1.0 / na, np.float32),
                "action_ev": np.arange(na * nh[p], dtype=np.float32).reshape(na, nh[p])}
    gpu = g.GpuSolver.__new__(g.GpuSolver)
    gpu._h = None
    gpu.solver = sv
    gpu.node_values = fake_values
    v = gpu.node_view(path)
    assert set(v) == {"node_type", "street", "board", "pot", "put", "player", "actions", "available_cards", "players",
                      "locked", "history"}
    assert v["actions"] == hv["actions"] and v["history"] == hv["history"]
    for q in (0, 1):
        hands = v["players"][q]["hands"]
        assert len(hands) == nh[q]
        c1, c2, w, _ = spot.hands(q)
        h0 = hands[0]
        assert h0["combo"] == g.combo_string(int(c1[0]), int(c2[0])) and len(h0["combo"]) == 4
        assert h0["weight"] == float(w[0]) and h0["reach"] == 0.5 and h0["valid"] == 2.0
        assert (h0["eq"] is None) == (q == 1)
        if q == p:
            assert h0["ev"] is None and len(h0["strategy"]) == na and len(h0["evs"]) == na
            assert hands[1]["evs"] == [float(a * nh[p] + 1) for a in range(na)]
        else:
            assert "strategy" not in h0 and "evs" not in h0 and h0["ev"] == 1.0
    # combo strings: higher rank first, on equal ranks the higher suit first
    assert g.combo_string(0, 51) == "As2c" and g.combo_string(48, 51) == "AsAc"


def _stub_gpu(sv, **methods):
    gpu = g.GpuSolver.__new__(g.GpuSolver)
    gpu._h = None
    gpu.solver = sv
    for k, f in methods.items():
        setattr(gpu, k, f)
    return gpu


def test_exploit_view_and_runouts_report_compose():
    """GpuSolver.exploit_view and runouts_report assembled from stand-in
    device numbers: the reference's ExploitView and RunoutsReport fields."""
    cfg = W.small_flop_spot()
    spot = g.Spot(cfg)
    sv = g.Solver(spot)
    hv = sv.path_view([1])
    na, p = len(hv["actions"]), hv["player"]
    nh = spot.nh[p]

    def fake_exploit(path, exploiter, solver=None):
        z = np.ones(spot.nh[exploiter], np.float32)
        gain = z.copy()
        gain[0] = np.nan
        return {"node": hv["node"], "kind": 0, "player": p, "reach": z, "valid": z * 2, "br_ev": z * 3,
                "cur_ev": z * 2, "gain": gain, "averages": np.array([3, 2, np.nan], np.float32),
                "br_strategy": np.eye(na, nh, dtype=np.float32), "action_ev": np.zeros((na, nh), np.float32)}
    gpu = _stub_gpu(sv, exploit_values=fake_exploit)
    ev = gpu.exploit_view([1], p)
    assert set(ev) == {"node_type", "exploiter", "player", "actions", "locked", "hands", "avg_br_ev", "avg_cur_ev",
                       "avg_gain"}
    assert ev["actions"] == hv["actions"] and ev["avg_gain"] is None and ev["avg_br_ev"] == 3.0
    assert ev["hands"][0]["gain"] is None and ev["hands"][0]["br_strategy"] == [1.0] + [0.0] * (na - 1)
    other = gpu.exploit_view([1], 1 - p)
    assert "br_strategy" not in other["hands"][0]

    chance = [0, 0]  # check, check: the turn's chance node
    cv = sv.path_view(chance)
    assert cv["node_type"] == "chance"
    cards = [("23456789TJQKA".index(c[0]) * 4 + "cdhs".index(c[1])) for c in cv["available_cards"]][::-1]

    def fake_runouts(path, solver=None):
        rows = [{"card": c, "freqs": np.full(2, 0.5, np.float32), "eq": [0.4, np.nan], "ev": [1.0, 2.0]}
                for c in cards]
        return {"player": 0, "num_actions": 2, "pot": 60.0, "rows": rows}
    rep = _stub_gpu(sv, runouts=fake_runouts).runouts_report(chance)
    assert rep["pot"] == 60.0 and rep["player"] == 0 and len(rep["rows"]) == len(cards)
    assert rep["rows"][0]["card"] == g.card_string(cards[0]) and rep["rows"][0]["eq"] == [pytest.approx(0.4), None]
    assert rep["actions"] == sv.path_view(chance + [g.card_string(cards[0])])["actions"]


def test_stack_sized_turn_bet_is_labelled_all_in():
    """The reference's runouts_labels_allin_bets (tests/convergence.rs:847-873)
    on the host side: on Th9h2c with 60 behind and a 60%-pot turn bet, the
    turn node after the report's first card (the highest available) offers
    the bet labelled "All-in" -- the label the runouts report copies from
    that node's action bar."""
    empty = {"bet": [], "raise": []}
    cfg = {"board": "Th9h2c", "range_oop": "QQ,JJ,TT", "range_ip": "AA,KK",
           "tree": {"starting_pot": 100.0, "effective_stack": 60.0,
                    "oop": [dict(empty), {"bet": W.sizes("60"), "raise": []}, dict(empty)],
                    "ip": [dict(empty), dict(empty), dict(empty)]}}
    sv = g.Solver(g.Spot(cfg))
    chance = [0, 0]
    cv = sv.path_view(chance)
    assert cv["node_type"] == "chance"
    first = cv["available_cards"][-1]  # the report's rows run from the highest card down
    labels = [a["label"] for a in sv.path_view(chance + [first])["actions"]]
    assert labels == ["Check", "All-in 60"], labels
