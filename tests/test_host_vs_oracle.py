"""Host side of the product (libgtob's C++ core, through the C ABI) against
the CPU oracle: tree construction (tree.rs), hand lists and same-combo maps
(game.rs:400-470), suit symmetries (iso.rs), river tables (game.rs:490-560),
pair weight sums (best_response.rs:240-252), arena codecs (store.rs),
locks (query.rs:700-773), the save format (persist.rs) and the exported
symbol set of include/gtob.h.  None of these tests needs a GPU.
"""
import ctypes
import json
import os
import re

import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench_spot():
    with open(os.path.join(ROOT, "tests", "golden", "bench_spot.json")) as f:
        return json.load(f)


def _allin_spot():
    cfg = W.small_flop_spot()
    for st in cfg["tree"]["oop"] + cfg["tree"]["ip"]:
        st["bet"] = [{"PotPct": 75.0}, "AllIn"]
        st["raise"] = ["AllIn"]
    cfg["tree"]["effective_stack"] = 120.0
    return cfg


def _raked_spot():
    cfg = W.small_flop_spot()
    cfg["tree"]["rake_pct"] = 0.05
    cfg["tree"]["rake_cap"] = 3.0
    return cfg


SPOTS = {
    "clairvoyance": W.clairvoyance_spot,
    "small_flop": W.small_flop_spot,
    "river": W.river_spot,
    "turn": lambda: W.turn_spot(g.evaluate7),
    "iso": W.iso_spot,
    "allin": _allin_spot,
    "raked": _raked_spot,
}


@pytest.fixture(scope="module", params=sorted(SPOTS))
def pair(request):
    cfg = SPOTS[request.param]()
    return request.param, po.Spot(cfg), g.Spot(cfg)


def test_tree_identical(pair):
    name, o, s = pair
    assert o.num_nodes == s.num_nodes, name
    a, b = o.nodes(), s.tree()
    for k in a:
        assert np.array_equal(a[k], b[k]), (name, k)
    assert np.array_equal(o.children(), s.children())
    ka, aa = o.actions()
    kb, ab = s.actions()
    assert np.array_equal(ka, kb) and np.array_equal(aa, ab)
    assert o.data_size == s.data_size


def test_hands_and_same_combo_identical(pair):
    name, o, s = pair
    for p in (0, 1):
        c1, c2, w = o.hands(p)
        d1, d2, dw, same = s.hands(p)
        assert np.array_equal(c1, d1) and np.array_equal(c2, d2), (name, p)
        assert np.array_equal(w, dw), (name, p)
        assert np.array_equal(o.same_combo(p), same), (name, p)


def test_suit_perms_identical(pair):
    name, o, s = pair
    assert o.num_perms == s.num_suit_perms
    for x, y in zip(o.perms(), s.suit_perms()):
        assert np.array_equal(x, y), name


def test_pair_weight_sum_identical(pair):
    name, o, s = pair
    assert o.pair_weight_sum() == s.pair_weight_sum(), name


def _river_keys(board_len, board, rng, n):
    live = [c for c in range(52) if c not in board]
    if board_len == 5:
        return [[]]
    if board_len == 4:
        return [[c] for c in live]
    keys = []
    for _ in range(n):
        t, r = rng.choice(live, 2, replace=False)
        keys.append([int(t), int(r)])
    return keys


def _board_cards(text):
    return ["23456789TJQKA".index(text[i].upper()) * 4 + "cdhs".index(text[i + 1].lower())
            for i in range(0, len(text), 2)]


def test_river_tables_identical(pair):
    name, o, s = pair
    board = _board_cards(s.config["board"])
    rng = np.random.default_rng(7)
    for dealt in _river_keys(len(board), board, rng, 40):
        for p in (0, 1):
            st0, ix0 = o.river(p, dealt)
            st1, ix1 = s.river(p, dealt)
            assert np.array_equal(st0, st1) and np.array_equal(ix0, ix1), (name, dealt, p)


def test_bench_spot_host_structures_identical():
    cfg = _bench_spot()
    o, s = po.Spot(cfg), g.Spot(cfg)
    assert o.num_nodes == s.num_nodes
    a, b = o.nodes(), s.tree()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    for p in (0, 1):
        assert np.array_equal(o.same_combo(p), s.hands(p)[3])
    for x, y in zip(o.perms(), s.suit_perms()):
        assert np.array_equal(x, y)


def test_evaluator_and_ranges_match_oracle():
    rng = np.random.default_rng(11)
    L = po.lib()
    for _ in range(3000):
        cards = rng.choice(52, 7, replace=False).astype(np.uint8)
        assert g.evaluate7(cards) == L.orc_evaluate7(po.ptr(cards))
    for text in ("AA,KK,QQ", "AKs,AQo:0.5", "22+,A2s+", "T9s-65s", "KQ,KJ:0.25", "AhKh,QcQd"):
        assert np.array_equal(g.parse_range(text), _oracle_range(text)), text


def _oracle_range(text):
    out = np.zeros(1326, np.float32)
    rc = po.lib().orc_parse_range(text.encode(), po.ptr(out))
    assert rc == 0
    return out


@pytest.mark.parametrize("storage", ["f32", "compressed"])
def test_arena_codecs_match_oracle(storage):
    """set_arena -> arena: f32 is the identity; compressed encodes each node
    with store.rs's per-node scale and decodes it again."""
    cfg = W.small_flop_spot()
    o, s = po.Spot(cfg), g.Spot(cfg)
    osv = po.Solver(o, compressed=storage != "f32")
    hsv = g.Solver(s, storage=storage)
    rng = np.random.default_rng(5)
    for which in (0, 1):
        for p in (0, 1):
            x = rng.standard_normal(s.data_size[p]).astype(np.float32) * 40.0
            if which == 1:
                x = np.abs(x)
            x[rng.random(x.size) < 0.05] = 0.0
            osv.set_arena(which, p, x)
            hsv.set_arena(which, p, x)
            a, b = osv.arena(which, p), hsv.arena(which, p)
            assert np.array_equal(a, b), (storage, which, p)
            if storage == "f32":
                assert np.array_equal(b, x)


def _seed_regrets(osv, hsv, spot, seed):
    rng = np.random.default_rng(seed)
    for which in (0, 1):
        for p in (0, 1):
            x = np.abs(rng.standard_normal(spot.data_size[p]).astype(np.float32)) * 3.0
            if which == 0:
                x -= 1.5
            osv.set_arena(which, p, x)
            hsv.set_arena(which, p, x)


def test_locks_match_oracle():
    cfg = W.small_flop_spot()
    o, s = po.Spot(cfg), g.Spot(cfg)
    osv = po.Solver(o, use_iso=False)
    hsv = g.Solver(s, use_iso=False)
    _seed_regrets(osv, hsv, s, 3)
    t = s.tree()
    root_na = int(t["nchild"][0])
    # freeze at the root: the current solved strategy becomes the lock
    n0 = osv.lock_node([], 0)
    n1 = hsv.lock_node([], "freeze")
    assert n0 == n1 == 0
    na, nh = root_na, s.nh[0]
    assert np.array_equal(osv.solved_strategy(0, na, nh), hsv.solved_strategy(0))
    # a range-wide frequency lock one step down (the IP node after a check)
    freqs = [0.25] + [0.75 / (int(t["nchild"][int(s.children()[t["child_start"][0]])]) - 1)] * (
        int(t["nchild"][int(s.children()[t["child_start"][0]])]) - 1)
    n0 = osv.lock_node([0], 1, freqs=freqs)
    n1 = hsv.lock_node([0], "range", freqs=freqs)
    assert n0 == n1
    na1, nh1 = int(t["nchild"][n1]), s.nh[int(t["player"][n1])]
    assert np.array_equal(osv.solved_strategy(n0, na1, nh1), hsv.solved_strategy(n1))
    assert hsv.num_locks == 2


def test_save_load_roundtrip(tmp_path):
    """persist.rs: magic, JSON header line, then raw f32 arenas; the loaded
    solver rebuilds the spot and gets the same arenas, iteration and locks."""
    cfg = W.small_flop_spot()
    s = g.Spot(cfg)
    hsv = g.Solver(s)
    rng = np.random.default_rng(9)
    arenas = {}
    for which in (0, 1):
        for p in (0, 1):
            x = rng.standard_normal(s.data_size[p]).astype(np.float32)
            hsv.set_arena(which, p, x)
            arenas[which, p] = x
    hsv.iteration = 123
    hsv.lock_node([], "range", freqs=[1.0] + [0.0] * (int(s.tree()["nchild"][0]) - 1), label="always check")
    path = tmp_path / "spot.gto"
    hsv.save(path)
    raw = path.read_bytes()
    assert raw[:10] == b"GTOSOLVE2\n"  # persist.rs magic
    nl = raw.index(b"\n", 10)
    header = json.loads(raw[10:nl])
    assert header["iteration"] == 123
    assert header["config"]["board"] == cfg["board"]
    # body: regrets[0], regrets[1], strategy[0], strategy[1], each a u64 LE
    # length followed by that many f32 (persist.rs:60-95)
    pos = nl + 1
    for k in range(4):
        p, which = k % 2, 0 if k < 2 else 1
        n = int.from_bytes(raw[pos:pos + 8], "little")
        assert n == s.data_size[p]
        arr = np.frombuffer(raw, np.float32, n, pos + 8)
        assert np.array_equal(arr, arenas[which, p]), (which, p)
        pos += 8 + 4 * n
    assert pos == len(raw)
    back = g.Solver.load(path)
    assert back.iteration == 123
    assert back.num_locks == 1
    for (which, p), x in arenas.items():
        assert np.array_equal(back.arena(which, p), x), (which, p)


def _doctor_locks(path, locks):
    """Rewrite the header's lock list, arenas untouched (tests/save_locks.rs:60-70)."""
    raw = path.read_bytes()
    nl = raw.index(b"\n", 10)
    header = json.loads(raw[10:nl])
    header["locks"] = locks
    path.write_bytes(raw[:10] + json.dumps(header).encode() + raw[nl:])


@pytest.mark.parametrize("case", ["out_of_range", "non_action", "short_sigma", "negative"])
def test_load_rejects_bad_locks(tmp_path, case):
    """tests/save_locks.rs:100-163: malformed locks are refused at load."""
    cfg = W.small_flop_spot()
    s = g.Spot(cfg)
    hsv = g.Solver(s)
    path = tmp_path / "bad.gto"
    hsv.save(path)
    t = s.tree()
    n_root = int(t["nchild"][0]) * s.nh[int(t["player"][0])]
    if case == "out_of_range":
        locks, want = [[999999, [0.25] * 4]], "out of range"
    elif case == "non_action":
        idx = int(np.nonzero(t["kind"] != 0)[0][0])
        locks, want = [[idx, [0.5, 0.5]]], "not an action node"
    elif case == "short_sigma":
        locks, want = [[0, [0.5]]], "expected"
    else:
        sig = [0.5] * n_root
        sig[0] = -1.0
        locks, want = [[0, sig]], "finite"
    _doctor_locks(path, locks)
    with pytest.raises(g.GtobError) as e:
        g.Solver.load(path)
    assert want in str(e.value) and "lock" in str(e.value), str(e.value)


def test_lock_survives_save_load(tmp_path):
    """tests/save_locks.rs:72-97 on the product's save format."""
    s = g.Spot(W.small_flop_spot())
    hsv = g.Solver(s)
    rng = np.random.default_rng(2)
    hsv.set_arena(0, 0, rng.standard_normal(s.data_size[0]).astype(np.float32))
    hsv.lock_node([], "freeze", label="root")
    before = hsv.solved_strategy(0)
    path = tmp_path / "lock.gto"
    hsv.save(path)
    back = g.Solver.load(path)
    assert back.num_locks == 1
    assert np.array_equal(back.solved_strategy(0), before)


def test_c_abi_exports_every_declared_symbol():
    with open(os.path.join(ROOT, "include", "gtob.h")) as f:
        text = f.read()
    names = sorted(set(re.findall(r"\b(gtob_[a-z0-9_]+)\s*\(", text)))
    assert len(names) > 40
    lib = ctypes.CDLL(os.path.join(ROOT, "gtopen_b200", "libgtob.so"))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_invalid_inputs_are_errors_not_crashes():
    with pytest.raises(g.GtobError):
        g.Spot({"board": "XxYy"})
    with pytest.raises(g.GtobError):
        g.parse_range("AK:2.0:bad")
    s = g.Spot(W.small_flop_spot())
    hsv = g.Solver(s)
    with pytest.raises(g.GtobError):
        hsv.lock_node([99], "freeze")
    with pytest.raises(g.GtobError):
        hsv.set_lock(0, np.zeros(3, np.float32))


def test_batch_host_side():
    """A batch holds one host solver per spot before it runs; without a GPU
    the run is an error, not a crash."""
    spots = [g.Spot(W.small_flop_spot()), g.Spot(W.iso_spot())]
    b = g.Batch(spots, storage="compressed")
    assert [b.solver(i).iteration for i in range(2)] == [0, 0]
    assert b.solver(1).arena(1, 0).shape == (spots[1].data_size[0],)
    rows = b.rows()
    assert [r["iterations"] for r in rows] == [0, 0]
    if g.vram_info_mb() is None:
        with pytest.raises(g.GtobError) as e:
            b.run(max_iterations=5)
        assert "cuda" in str(e.value)


def test_canonical_flops_kat():
    """cards.rs:183-191: 1755 suit-isomorphism classes whose weights sum to
    the 22,100 flops."""
    classes = W.canonical_flops()
    assert len(classes) == 1755
    assert sum(w for _, w in classes) == 22100


@pytest.mark.parametrize("cfg_fn,use_iso", [(W.small_flop_spot, False), (W.iso_spot, True)])
@pytest.mark.parametrize("nshards", [2, 3])
def test_shard_partition(cfg_fn, use_iso, nshards):
    """A flop split by turn card: every shard keeps the tree above the first
    chance nodes, and every other visited node lies in exactly one shard."""
    spot = g.Spot(cfg_fn())
    full = g.shard_visited(spot, 0, 1, use_iso).astype(bool)
    parts = [g.shard_visited(spot, k, nshards, use_iso).astype(bool) for k in range(nshards)]
    union = np.logical_or.reduce(parts)
    common = np.logical_and.reduce(parts)
    assert np.array_equal(union, full)
    count = np.sum(parts, axis=0)
    assert np.array_equal(count[full & ~common], np.ones((full & ~common).sum()))
    assert common.sum() < full.sum() / 2  # the shared top part is small
    for k in range(nshards):
        assert (parts[k] & ~common).any()

