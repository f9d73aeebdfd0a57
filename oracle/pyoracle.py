"""ctypes binding of the CPU oracle (liboracle.so) -- test infrastructure only.

Used by tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
to check and time the product library.  Configs are the reference's
SpotConfig as a plain dict (the JSON schema of game.rs:22-27 / tree.rs:70-95).
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class Size(C.Structure):
    _fields_ = [("kind", C.c_int), ("value", C.c_double)]


class Config(C.Structure):
    _fields_ = [
        ("board", C.c_char_p), ("range_oop", C.c_char_p), ("range_ip", C.c_char_p),
        ("starting_pot", C.c_double), ("effective_stack", C.c_double), ("rake_pct", C.c_double),
        ("rake_cap", C.c_double), ("allin_threshold", C.c_double),
        ("add_allin", C.c_int), ("max_raises", C.c_int),
        ("n", C.c_int * 3 * 3 * 2),
        ("sizes", Size * 8 * 3 * 3 * 2),
    ]


def build():
    """Compile liboracle.so in place (g++ -fopenmp)."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.c_void_p
        L.orc_last_error.restype = C.c_char_p
        L.orc_evaluate7.restype = C.c_uint32
        L.orc_spot_new.restype = P
        L.orc_spot_new.argtypes = [C.POINTER(Config), C.c_int, C.c_uint64]
        for f in ("orc_spot_num_nodes", "orc_spot_num_children", "orc_spot_num_actions"):
            getattr(L, f).restype = C.c_int64
            getattr(L, f).argtypes = [P]
        L.orc_spot_data_size.restype = C.c_uint64
        L.orc_spot_data_size.argtypes = [P, C.c_int]
        L.orc_spot_num_hands.argtypes = [P, C.c_int]
        L.orc_spot_num_perms.argtypes = [P]
        L.orc_spot_free.argtypes = [P]
        L.orc_spot_nodes.argtypes = [P] + [P] * 12
        L.orc_spot_children.argtypes = [P, P]
        L.orc_spot_actions.argtypes = [P, P, P]
        L.orc_spot_hands.argtypes = [P, C.c_int, P, P, P]
        L.orc_spot_same_combo.argtypes = [P, C.c_int, P]
        L.orc_spot_perms.argtypes = [P, P, P, P]
        L.orc_spot_river.argtypes = [P, C.c_int, P, C.c_int, P, P]
        L.orc_spot_pair_weight_sum.restype = C.c_double
        L.orc_spot_pair_weight_sum.argtypes = [P]
        L.orc_fold_cfv.argtypes = [P, C.c_int, P, C.c_float, C.c_int, P]
        L.orc_showdown_cfv.argtypes = [P, C.c_int, P, C.c_int, P, C.c_float, C.c_float, C.c_float, C.c_int, P]
        L.orc_solver_set_sums.argtypes = [P, C.c_int]
        L.orc_solver_set_rounding.argtypes = [P, C.c_int]
        L.orc_solver_new.restype = P
        L.orc_solver_new.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_solver_free.argtypes = [P]
        L.orc_solver_iterate.argtypes = [P, C.c_int]
        L.orc_solver_iteration.restype = C.c_uint32
        L.orc_solver_iteration.argtypes = [P]
        L.orc_solver_set_iteration.argtypes = [P, C.c_uint32]
        L.orc_solver_exploitability.restype = C.c_double
        L.orc_solver_exploitability.argtypes = [P]
        L.orc_solver_exploitability_f64.restype = C.c_double
        L.orc_solver_exploitability_f64.argtypes = [P]
        L.orc_solver_get_arena.argtypes = [P, C.c_int, C.c_int, P]
        L.orc_solver_set_arena.argtypes = [P, C.c_int, C.c_int, P]
        L.orc_solver_set_lock.argtypes = [P, C.c_uint32, P, C.c_int]
        L.orc_solver_clear_locks.argtypes = [P]
        L.orc_solver_avg_strategy.argtypes = [P, C.c_uint32, P]
        L.orc_solver_solved_strategy.argtypes = [P, C.c_uint32, P]
        L.orc_solver_ensure_symmetric.argtypes = [P]
        L.orc_solver_root_br_cfv.argtypes = [P, C.c_int, P]
        L.orc_solver_discounts.argtypes = [C.c_int, C.c_uint32, P, P, P]
        L.orc_solver_walk_path.argtypes = [P, P, C.c_int, P, P, P]
        L.orc_solver_node_values.argtypes = [P, P, C.c_int, C.c_int, C.c_int, P, P, P, P]
        L.orc_solver_node_values.restype = C.c_int
        L.orc_rake_to_target.argtypes = [P, C.c_int, C.c_int, P, P]
        L.orc_normalize_freqs.argtypes = [P, C.c_int, P]
        L.orc_solver_lock_node.argtypes = [P, P, C.c_int, C.c_int, P, C.c_int, C.c_char_p]
        L.orc_encode_i16.restype = C.c_float
        L.orc_encode_i16.argtypes = [P, C.c_int, P]
        L.orc_encode_u16.restype = C.c_float
        L.orc_encode_u16.argtypes = [P, C.c_int, P]
        L.orc_decode_i16.argtypes = [P, C.c_int, C.c_float, P]
        L.orc_decode_u16.argtypes = [P, C.c_int, C.c_float, P]
        L.orc_parse_range.argtypes = [C.c_char_p, P]
        L.orc_parse_cards.argtypes = [C.c_char_p, P, C.c_int]
        L.orc_canonical_flops.argtypes = [P, P, C.c_int]
        L.orc_canonical_flops_subset.argtypes = [C.c_int, P, P, C.c_int]
        L.orc_straight_top.argtypes = [C.c_uint16]
        L.orc_ref_eval7.argtypes = [P, P, P, P]
        L.orc_set_threads.argtypes = [C.c_int]
        _LIB = L
    return _LIB


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


_KIND = {"PotPct": 0, "PrevMult": 1}


def evaluate7(cards):
    """7-card strength (evaluator.rs:68-174), the oracle's restatement."""
    c = np.ascontiguousarray(cards, np.uint8)
    return int(lib().orc_evaluate7(ptr(c)))


def make_config(cfg):
    """dict SpotConfig -> ctypes Config (keeps the byte strings alive on the object)."""
    c = Config()
    keep = [cfg["board"].encode(), cfg["range_oop"].encode(), cfg["range_ip"].encode()]
    c.board, c.range_oop, c.range_ip = keep
    t = cfg["tree"]
    c.starting_pot = float(t["starting_pot"])
    c.effective_stack = float(t["effective_stack"])
    c.rake_pct = float(t.get("rake_pct", 0.0))
    c.rake_cap = float(t.get("rake_cap", 0.0))
    c.allin_threshold = float(t.get("allin_threshold", 0.85))
    c.add_allin = int(bool(t.get("add_allin", False)))
    c.max_raises = int(t.get("max_raises", 10))
    for p, key in enumerate(("oop", "ip")):
        for s in range(3):
            st = t[key][s]
            for li, lname in enumerate(("bet", "raise", "donk")):
                lst = st.get(lname, [])
                if len(lst) > 8:
                    raise ValueError("at most 8 sizes per list")
                c.n[p][s][li] = len(lst)
                for k, sz in enumerate(lst):
                    if sz == "AllIn":
                        c.sizes[p][s][li][k].kind = 2
                        c.sizes[p][s][li][k].value = 0.0
                    else:
                        (name, v), = sz.items()
                        c.sizes[p][s][li][k].kind = _KIND[name]
                        c.sizes[p][s][li][k].value = float(v)
    c._keep = keep
    return c


class OracleError(RuntimeError):
    pass


class Spot:
    def __init__(self, cfg, lenient=False, max_nodes=0):
        L = lib()
        self._cfg = make_config(cfg)
        self.h = L.orc_spot_new(C.byref(self._cfg), int(lenient), int(max_nodes))
        if not self.h:
            raise OracleError(L.orc_last_error().decode())
        self.num_nodes = L.orc_spot_num_nodes(self.h)
        self.nh = [L.orc_spot_num_hands(self.h, 0), L.orc_spot_num_hands(self.h, 1)]
        self.data_size = [L.orc_spot_data_size(self.h, 0), L.orc_spot_data_size(self.h, 1)]
        self.num_perms = L.orc_spot_num_perms(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_spot_free(self.h)
            self.h = None

    def nodes(self):
        n = self.num_nodes
        out = dict(kind=np.zeros(n, np.uint8), player=np.zeros(n, np.uint8), street=np.zeros(n, np.uint8),
                   nchild=np.zeros(n, np.uint8), child_start=np.zeros(n, np.uint32),
                   action_start=np.zeros(n, np.uint32), data_off=np.zeros(n, np.uint64),
                   put0=np.zeros(n), put1=np.zeros(n), twin=np.zeros(n), tlose=np.zeros(n), ttie=np.zeros(n))
        lib().orc_spot_nodes(self.h, *[ptr(out[k]) for k in ("kind", "player", "street", "nchild", "child_start",
                                                              "action_start", "data_off", "put0", "put1", "twin",
                                                              "tlose", "ttie")])
        return out

    def children(self):
        a = np.zeros(lib().orc_spot_num_children(self.h), np.uint32)
        lib().orc_spot_children(self.h, ptr(a))
        return a

    def actions(self):
        n = lib().orc_spot_num_actions(self.h)
        k, amt = np.zeros(n, np.int32), np.zeros(n)
        lib().orc_spot_actions(self.h, ptr(k), ptr(amt))
        return k, amt

    def hands(self, p):
        n = self.nh[p]
        c1, c2, w = np.zeros(n, np.uint8), np.zeros(n, np.uint8), np.zeros(n, np.float32)
        lib().orc_spot_hands(self.h, p, ptr(c1), ptr(c2), ptr(w))
        return c1, c2, w

    def same_combo(self, p):
        a = np.zeros(self.nh[p], np.uint32)
        lib().orc_spot_same_combo(self.h, p, ptr(a))
        return a

    def perms(self):
        k = self.num_perms
        pm = np.zeros((k, 4), np.uint8)
        h0 = np.zeros((k, self.nh[0]), np.uint16)
        h1 = np.zeros((k, self.nh[1]), np.uint16)
        lib().orc_spot_perms(self.h, ptr(pm), ptr(h0), ptr(h1))
        return pm, h0, h1

    def river(self, p, dealt):
        d = np.array(dealt, np.uint8)
        st = np.zeros(self.nh[p], np.uint32)
        ix = np.zeros(self.nh[p], np.uint16)
        n = lib().orc_spot_river(self.h, p, ptr(d), len(dealt), ptr(st), ptr(ix))
        if n < 0:
            raise OracleError(lib().orc_last_error().decode())
        return st[:n], ix[:n]

    def pair_weight_sum(self):
        return lib().orc_spot_pair_weight_sum(self.h)

    def fold_cfv(self, p, reach_o, amount, exact=False):
        out = np.zeros(self.nh[p], np.float32)
        r = np.ascontiguousarray(reach_o, np.float32)
        lib().orc_fold_cfv(self.h, p, ptr(r), float(amount), int(exact), ptr(out))
        return out

    def showdown_cfv(self, p, dealt, reach_o, win, lose, tie, exact=False):
        out = np.zeros(self.nh[p], np.float32)
        r = np.ascontiguousarray(reach_o, np.float32)
        d = np.array(dealt, np.uint8)
        lib().orc_showdown_cfv(self.h, p, ptr(d), len(dealt), ptr(r), float(win), float(lose), float(tie),
                               int(exact), ptr(out))
        return out


ALGOS = {"dcfr": 0, "cfr+": 1, "pcfr+": 2}


class Solver:
    """The reference CPU engine (cfr.rs); prune=True reproduces it exactly,
    prune=False gives the no-pruning semantics of a level-synchronous sweep.
    exact=False sums terminal reach in f64 as the reference does (game.rs);
    exact=True uses the GPU engine's exact fixed-point terminal sums.
    stochastic=True requantises the 16-bit arenas with the engine's
    stochastic rounding instead of store.rs's round-to-nearest."""

    def __init__(self, spot, compressed=False, algo="dcfr", use_iso=True, prune=True, fp8=False, exact=False,
                 stochastic=False):
        self.spot = spot
        mode = 2 if fp8 else int(bool(compressed))
        self.h = lib().orc_solver_new(spot.h, mode, ALGOS[algo], int(use_iso), int(prune))
        if exact:
            lib().orc_solver_set_sums(self.h, 1)
        if stochastic:
            lib().orc_solver_set_rounding(self.h, 1)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_solver_free(self.h)
            self.h = None

    def iterate(self, n=1):
        lib().orc_solver_iterate(self.h, int(n))

    @property
    def iteration(self):
        return lib().orc_solver_iteration(self.h)

    @iteration.setter
    def iteration(self, v):
        lib().orc_solver_set_iteration(self.h, int(v))

    def exploitability(self):
        return lib().orc_solver_exploitability(self.h)

    def exploitability_f64(self):
        return lib().orc_solver_exploitability_f64(self.h)

    def arena(self, which, p):
        out = np.zeros(self.spot.data_size[p], np.float32)
        lib().orc_solver_get_arena(self.h, which, p, ptr(out))
        return out

    def set_arena(self, which, p, data):
        d = np.ascontiguousarray(data, np.float32)
        lib().orc_solver_set_arena(self.h, which, p, ptr(d))

    def set_lock(self, node, sigma):
        s = np.ascontiguousarray(sigma, np.float32)
        lib().orc_solver_set_lock(self.h, int(node), ptr(s), s.size)

    def avg_strategy(self, node, na, nh):
        out = np.zeros(na * nh, np.float32)
        lib().orc_solver_avg_strategy(self.h, int(node), ptr(out))
        return out

    def solved_strategy(self, node, na, nh):
        out = np.zeros(na * nh, np.float32)
        lib().orc_solver_solved_strategy(self.h, int(node), ptr(out))
        return out

    def ensure_symmetric(self):
        lib().orc_solver_ensure_symmetric(self.h)

    def root_br_cfv(self, p):
        out = np.zeros(self.spot.nh[p], np.float32)
        lib().orc_solver_root_br_cfv(self.h, p, ptr(out))
        return out

    def node_values(self, steps, p, na_max=8, avg=True):
        """query.rs node_view's (avg) or exploit_view's (best response)
        traversals for player p at the node `steps` reaches (actions >= 0,
        cards as -1 - card): (node, cfv, child cfvs (na_max x nh, rows of p's
        actions when p acts), reach0, reach1)."""
        st = np.array(list(steps) + [0], np.int32)
        h = self.spot.nh[p]
        cfv = np.zeros(h, np.float32)
        child = np.zeros((na_max, h), np.float32)
        r0 = np.zeros(self.spot.nh[0], np.float32)
        r1 = np.zeros(self.spot.nh[1], np.float32)
        n = lib().orc_solver_node_values(self.h, ptr(st), len(steps), p, int(avg), ptr(cfv), ptr(child), ptr(r0),
                                         ptr(r1))
        if n < 0:
            raise RuntimeError("oracle node_values failed")
        return n, cfv, child, r0, r1

    def lock_node(self, steps, mode, freqs=None, combo=""):
        st = np.array(steps if steps else [0], np.int32)
        fr = np.array(freqs if freqs is not None else [0.0], np.float32)
        r = lib().orc_solver_lock_node(self.h, ptr(st), len(steps), int(mode), ptr(fr),
                                       len(freqs) if freqs is not None else 0, combo.encode())
        if r < 0:
            raise OracleError(lib().orc_last_error().decode())
        return r


def discounts(algo, t):
    a, b, c = C.c_float(), C.c_float(), C.c_float()
    lib().orc_solver_discounts(ALGOS[algo], int(t), C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


def fp8_encode(x):
    """FP8 E4M3 bytes of float32 values (round to nearest even, saturating)."""
    a = np.ascontiguousarray(x, np.float32)
    out = np.zeros(a.size, np.uint8)
    lib().orc_fp8_encode(ptr(a), a.size, ptr(out))
    return out


def fp8_decode(q):
    a = np.ascontiguousarray(q, np.uint8)
    out = np.zeros(a.size, np.float32)
    lib().orc_fp8_decode(ptr(a), a.size, ptr(out))
    return out


def set_threads(n):
    lib().orc_set_threads(int(n))
