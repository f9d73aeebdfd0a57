"""gtopen_b200 -- B200 discounted-CFR engine for heads-up postflop spots.

Python mirror of the reference solver crate's API for the GPU hot path
(MatthewPDingle/GTOpen crates/solver: game.rs Spot, cfr.rs Solver state,
gpu/mod.rs GpuSolver, save.rs), bound over the C ABI in include/gtob.h
(libgtob.so, built in place by gtopen_b200/csrc/Makefile).  There is no CPU
fallback: every call goes through libgtob, and importing the bindings fails
loudly if the library is missing.
"""
import ctypes as C
import json
import os

import numpy as np

__all__ = ["Spot", "Solver", "GpuSolver", "GtobError", "KERNEL_NAMES", "estimate_vram", "vram_info_mb",
           "evaluate7", "parse_range", "lib", "LIB_PATH"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgtob.so")
_LIB = None

STORAGE = {"f32": 0, "compressed": 1, "i16": 1}
ALGO = {"dcfr": 0, "cfr+": 1, "cfrplus": 1, "pcfr+": 2, "pcfrplus": 2}
DEVICE_FORMAT = {None: -1, "follow": -1, "f32": 0, "i16": 1, "fp8": 2, "i16sr": 3}
NODE_SCRATCH_ELEMS = 16384  # GTOB_NODE_SCRATCH_ELEMS
KERNEL_NAMES = ["copy_root", "down_action", "down_chance", "up_fold", "up_show", "up_chance", "up_action"]


class GtobError(RuntimeError):
    """A failed libgtob call (the reference's Result::Err(String))."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class SpotInfo(C.Structure):
    _fields_ = [("num_nodes", C.c_uint64), ("num_action_nodes", C.c_uint64), ("num_children", C.c_uint64),
                ("num_actions", C.c_uint64), ("data_size", C.c_uint64 * 2), ("num_hands", C.c_uint32 * 2),
                ("root_street", C.c_uint32), ("num_suit_perms", C.c_uint32)]


class GpuInfo(C.Structure):
    _fields_ = [("device_bytes", C.c_uint64), ("visited_nodes", C.c_uint64), ("cfv_slots", C.c_uint64),
                ("reach_slots", C.c_uint64 * 2), ("device_action_nodes", C.c_uint64 * 2),
                ("visited_terminals", C.c_uint64), ("num_levels", C.c_uint32), ("num_river_slots", C.c_uint32),
                ("arena_format", C.c_int32), ("iter_bytes", C.c_double), ("upload_bytes", C.c_uint64),
                ("iteration_kernels", C.c_uint32), ("river_programs", C.c_uint32)]


class NodeInfo(C.Structure):
    _fields_ = [("node", C.c_uint32), ("kind", C.c_int32), ("player", C.c_int32), ("num_actions", C.c_int32)]


class RunoutRow(C.Structure):
    _fields_ = [("card", C.c_int32), ("eq", C.c_float * 2), ("ev", C.c_float * 2)]


class BatchRow(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_uint32), ("exploit_pct", C.c_double),
                ("seconds", C.c_double), ("ev", C.c_double * 2)]


class BatchStats(C.Structure):
    _fields_ = [("launches", C.c_uint64), ("kernel_ms", C.c_double), ("tuned", C.c_int32), ("tile", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("grid", C.c_int32)]


# gtob_reduce_fn: int (*)(void* user, float* values, size_t count)
REDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_float), C.c_size_t)


class Profile(C.Structure):
    _fields_ = [("ms", C.c_double * 7), ("launches", C.c_uint32 * 7)]

    def as_dict(self):
        return {KERNEL_NAMES[k]: (self.ms[k], self.launches[k]) for k in range(7)}


def lib():
    """Load libgtob.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError("libgtob.so is not built: run `make -C gtopen_b200/csrc` (or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    P, I, U32, U64, D = C.c_void_p, C.c_int, C.c_uint32, C.c_uint64, C.c_double
    sig = {
        "gtob_last_error": (C.c_char_p, []),
        "gtob_kernel_name": (C.c_char_p, [I]),
        "gtob_version": (C.c_char_p, []),
        "gtob_spot_from_json": (I, [C.c_char_p, U64, I, C.POINTER(P)]),
        "gtob_spot_free": (None, [P]),
        "gtob_spot_info_get": (I, [P, C.POINTER(SpotInfo)]),
        "gtob_spot_tree": (I, [P] + [P] * 12),
        "gtob_spot_children": (I, [P, P]),
        "gtob_spot_actions": (I, [P, P, P]),
        "gtob_spot_hands": (I, [P, I, P, P, P, P]),
        "gtob_spot_suit_perms": (I, [P, P, P, P]),
        "gtob_spot_river": (I, [P, I, P, I, P, P]),
        "gtob_spot_pair_weight_sum": (D, [P]),
        "gtob_evaluate7": (U32, [P]),
        "gtob_parse_range": (I, [C.c_char_p, P]),
        "gtob_estimate_vram": (U64, [P]),
        "gtob_vram_info_mb": (I, [C.POINTER(U64), C.POINTER(U64)]),
        "gtob_solver_new": (I, [P, I, I, I, C.POINTER(P)]),
        "gtob_solver_free": (None, [P]),
        "gtob_solver_iteration": (U32, [P]),
        "gtob_solver_set_iteration": (I, [P, U32]),
        "gtob_solver_arena_bytes": (U64, [P]),
        "gtob_solver_get_arena": (I, [P, I, I, P]),
        "gtob_solver_set_arena": (I, [P, I, I, P]),
        "gtob_solver_average_strategy": (I, [P, U32, P]),
        "gtob_solver_solved_strategy": (I, [P, U32, P]),
        "gtob_solver_lock_node": (I, [P, P, I, I, P, I, C.c_char_p, C.c_char_p, C.POINTER(U32)]),
        "gtob_solver_set_lock": (I, [P, U32, P, U64, C.c_char_p]),
        "gtob_solver_clear_locks": (I, [P]),
        "gtob_solver_num_locks": (I, [P]),
        "gtob_solver_ensure_symmetric": (I, [P]),
        "gtob_save": (I, [P, C.c_char_p]),
        "gtob_load": (I, [C.c_char_p, I, C.POINTER(P)]),
        "gtob_gpu_new": (I, [P, I, C.POINTER(P)]),
        "gtob_gpu_new_ex": (I, [P, I, I, C.POINTER(P)]),
        "gtob_gpu_free": (None, [P]),
        "gtob_gpu_iterate": (I, [P, I]),
        "gtob_gpu_iterate_profiled": (I, [P, C.POINTER(Profile)]),
        "gtob_gpu_exploitability": (I, [P, P, C.POINTER(D)]),
        "gtob_gpu_sync_to_cpu": (I, [P, P]),
        "gtob_gpu_sync_strategy": (I, [P, P]),
        "gtob_gpu_synchronize": (I, [P]),
        "gtob_gpu_update_locks": (I, [P, P]),
        "gtob_gpu_iteration": (U32, [P]),
        "gtob_gpu_info_get": (I, [P, C.POINTER(GpuInfo)]),
        "gtob_gpu_root_cfv": (I, [P, I, I, P]),
        "gtob_gpu_export_arena": (I, [P, I, I, P]),
        "gtob_gpu_read_node_static": (I, [P, I, C.c_uint32, P, C.c_uint64, P]),
        "gtob_gpu_discounts": (I, [P, P]),
        "gtob_gpu_save": (I, [P, P, C.c_char_p]),
        "gtob_gpu_node_values": (I, [P, P, P, I, C.POINTER(NodeInfo)] + [P] * 10),
        "gtob_gpu_runouts": (I, [P, P, P, I, C.POINTER(RunoutRow), P, I, I, C.POINTER(I), C.POINTER(I), C.POINTER(I),
                                 C.POINTER(D)]),
        "gtob_gpu_exploit_values": (I, [P, P, P, I, I, C.POINTER(NodeInfo)] + [P] * 8),
        "gtob_batch_new": (I, [C.POINTER(P), I, I, I, I, I, I, I, C.POINTER(P)]),
        "gtob_nccl_unique_id": (I, [P]),
        "gtob_solver_path_view": (I, [P, P, I, C.c_char_p, U64, C.POINTER(U64)]),
        "gtob_gpu_new_sharded": (I, [P, I, I, I, I, P, C.POINTER(P)]),
        "gtob_gpu_new_sharded_host": (I, [P, I, I, I, I, REDUCE_FN, P, C.POINTER(P)]),
        "gtob_shards_new": (I, [P, I, I, I, C.POINTER(P)]),
        "gtob_shards_iterate": (I, [P, I]),
        "gtob_shards_exploitability": (I, [P, P, C.POINTER(D)]),
        "gtob_shards_export_arena": (I, [P, I, I, P]),
        "gtob_shards_sync_to_cpu": (I, [P, P, I]),
        "gtob_shards_free": (None, [P]),
        "gtob_spot_shard_visited": (I, [P, I, I, I, P]),
        "gtob_spot_batch_queue": (I, [C.POINTER(P), I, I, I, P, I, C.POINTER(I), C.POINTER(U64), C.POINTER(U64)]),
        "gtob_batch_run": (I, [P, U32, D, U32, I]),
        "gtob_batch_run_persistent": (I, [P, U32, D, U32, I]),
        "gtob_batch_stats_get": (I, [P, C.POINTER(BatchStats)]),
        "gtob_batch_size": (I, [P]),
        "gtob_batch_row_get": (I, [P, I, C.POINTER(BatchRow)]),
        "gtob_batch_root_cfv": (I, [P, I, I, P, I, C.POINTER(I)]),
        "gtob_batch_error": (C.c_char_p, [P, I]),
        "gtob_batch_solver": (P, [P, I]),
        "gtob_batch_free": (None, [P]),
        "gtob_gpu_load": (I, [C.c_char_p, I, I, I, C.POINTER(P), C.POINTER(P)]),
        "gtob_set_device": (I, [I]),
        "gtob_gpu_time_iterations": (I, [P, I, C.POINTER(D)]),
        "gtob_net_new": (I, [I, I, I, I, U64, C.POINTER(P)]),
        "gtob_net_free": (None, [P]),
        "gtob_net_get_params": (I, [P, I, P, P]),
        "gtob_net_set_params": (I, [P, I, P, P]),
        "gtob_net_get_grads": (I, [P, I, P, P]),
        "gtob_net_forward": (I, [P, P, I, P]),
        "gtob_net_gradients": (I, [P, P, P, P, I, C.POINTER(D)]),
        "gtob_net_train": (I, [P, P, P, P, I, I, I, C.c_float, U64, P]),
        "gtob_gemm_bf16": (I, [P, P, I, I, I, P]),
        "gtob_gpu_new_dl": (I, [P, P, I, I, C.POINTER(P)]),
        "gtob_gpu_leaves": (I, [P, P, P, P, I, C.POINTER(I)]),
        "gtob_spot_dl_plan": (I, [P, P, P, P, I, C.POINTER(I), P]),
        "gtob_gpu_node_sweep": (I, [P, U32, I, I, P, P, P]),
        "gtob_gpu_node_strategy": (I, [P, U32, P]),
        "gtob_gemm_time": (I, [I, I, I, I, C.POINTER(D)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(rc):
    if rc < 0:
        raise GtobError(rc, lib().gtob_last_error().decode(errors="replace"))
    return rc


def evaluate7(cards):
    c = np.ascontiguousarray(cards, np.uint8)
    return int(lib().gtob_evaluate7(_ptr(c)))


def parse_range(text):
    w = np.zeros(1326, np.float32)
    _check(lib().gtob_parse_range(text.encode(), _ptr(w)))
    return w


class Spot:
    """game.rs Spot: tree, hand lists, river tables, suit symmetries."""

    def __init__(self, config, max_nodes=0, lenient=False):
        text = config if isinstance(config, str) else json.dumps(config)
        h = C.c_void_p()
        _check(lib().gtob_spot_from_json(text.encode(), int(max_nodes), int(lenient), C.byref(h)))
        self._h = h
        self.config = json.loads(text)
        info = SpotInfo()
        _check(lib().gtob_spot_info_get(self._h, C.byref(info)))
        self.num_nodes = info.num_nodes
        self.num_action_nodes = info.num_action_nodes
        self.num_children = info.num_children
        self.num_actions = info.num_actions
        self.data_size = [info.data_size[0], info.data_size[1]]
        self.nh = [info.num_hands[0], info.num_hands[1]]
        self.root_street = info.root_street
        self.num_suit_perms = info.num_suit_perms

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.gtob_spot_free(self._h)
            self._h = None

    def tree(self):
        n = self.num_nodes
        out = dict(kind=np.zeros(n, np.uint8), player=np.zeros(n, np.uint8), street=np.zeros(n, np.uint8),
                   nchild=np.zeros(n, np.uint8), child_start=np.zeros(n, np.uint32),
                   action_start=np.zeros(n, np.uint32), data_off=np.zeros(n, np.uint64),
                   put0=np.zeros(n), put1=np.zeros(n), twin=np.zeros(n), tlose=np.zeros(n), ttie=np.zeros(n))
        keys = ("kind", "player", "street", "nchild", "child_start", "action_start", "data_off", "put0", "put1",
                "twin", "tlose", "ttie")
        _check(lib().gtob_spot_tree(self._h, *[_ptr(out[k]) for k in keys]))
        return out

    def children(self):
        a = np.zeros(self.num_children, np.uint32)
        _check(lib().gtob_spot_children(self._h, _ptr(a)))
        return a

    def actions(self):
        k = np.zeros(self.num_actions, np.int32)
        amt = np.zeros(self.num_actions)
        _check(lib().gtob_spot_actions(self._h, _ptr(k), _ptr(amt)))
        return k, amt

    def hands(self, p):
        n = self.nh[p]
        c1, c2 = np.zeros(n, np.uint8), np.zeros(n, np.uint8)
        w, same = np.zeros(n, np.float32), np.zeros(n, np.uint32)
        _check(lib().gtob_spot_hands(self._h, p, _ptr(c1), _ptr(c2), _ptr(w), _ptr(same)))
        return c1, c2, w, same

    def suit_perms(self):
        k = self.num_suit_perms
        pm = np.zeros((k, 4), np.uint8)
        h0, h1 = np.zeros((k, self.nh[0]), np.uint16), np.zeros((k, self.nh[1]), np.uint16)
        _check(lib().gtob_spot_suit_perms(self._h, _ptr(pm), _ptr(h0), _ptr(h1)))
        return pm, h0, h1

    def river(self, p, dealt):
        d = np.array(list(dealt) + [0, 0], np.uint8)
        st, ix = np.zeros(self.nh[p], np.uint32), np.zeros(self.nh[p], np.uint16)
        n = _check(lib().gtob_spot_river(self._h, p, _ptr(d), len(dealt), _ptr(st), _ptr(ix)))
        return st[:n], ix[:n]

    def pair_weight_sum(self):
        return lib().gtob_spot_pair_weight_sum(self._h)

    def estimate_vram(self):
        return int(lib().gtob_estimate_vram(self._h))


def estimate_vram(spot):
    return spot.estimate_vram()


def vram_info_mb():
    f, t = C.c_uint64(), C.c_uint64()
    if lib().gtob_vram_info_mb(C.byref(f), C.byref(t)) != 0:
        return None
    return f.value, t.value


class Solver:
    """cfr.rs Solver state: arenas, locks, iteration (the CFR loop runs on the GPU)."""

    def __init__(self, spot, storage="f32", algo="dcfr", use_iso=True, _handle=None):
        self.spot = spot
        self.storage = storage
        self.algo = algo
        if _handle is not None:
            self._h = _handle
            return
        h = C.c_void_p()
        _check(lib().gtob_solver_new(spot._h, STORAGE[storage], ALGO[algo], int(use_iso), C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None and getattr(self, "_owner", None) is None:
            _LIB.gtob_solver_free(self._h)
        self._h = None

    @property
    def iteration(self):
        return int(lib().gtob_solver_iteration(self._h))

    @iteration.setter
    def iteration(self, v):
        _check(lib().gtob_solver_set_iteration(self._h, int(v)))

    def arena_bytes(self):
        return int(lib().gtob_solver_arena_bytes(self._h))

    def arena(self, which, p):
        out = np.zeros(self.spot.data_size[p], np.float32)
        _check(lib().gtob_solver_get_arena(self._h, int(which), int(p), _ptr(out)))
        return out

    def set_arena(self, which, p, data):
        d = np.ascontiguousarray(data, np.float32)
        assert d.size == self.spot.data_size[p]
        _check(lib().gtob_solver_set_arena(self._h, int(which), int(p), _ptr(d)))

    def _na_nh(self, node):
        t = self.spot.tree()
        return int(t["nchild"][node]), self.spot.nh[int(t["player"][node])]

    def average_strategy(self, node, na=None, nh=None):
        if na is None:
            na, nh = self._na_nh(node)
        out = np.zeros(na * nh, np.float32)
        _check(lib().gtob_solver_average_strategy(self._h, int(node), _ptr(out)))
        return out

    def solved_strategy(self, node, na=None, nh=None):
        if na is None:
            na, nh = self._na_nh(node)
        out = np.zeros(na * nh, np.float32)
        _check(lib().gtob_solver_solved_strategy(self._h, int(node), _ptr(out)))
        return out

    def lock_node(self, path, mode, freqs=None, edits=None, label=""):
        """query.rs lock_node. path: list of ints (action index) or card strings;
        mode: "freeze" | "range" | "hands"."""
        steps = []
        for s in path:
            if isinstance(s, str):
                r, su = "23456789TJQKA".index(s[0].upper()), "cdhs".index(s[1].lower())
                steps.append(-1 - (r * 4 + su))
            else:
                steps.append(int(s))
        st = np.array(steps + [0], np.int32)
        m = {"freeze": 0, "range": 1, "hands": 2}[mode]
        fr = np.array((freqs or []) + [0.0], np.float32)
        ej = json.dumps([[c, list(map(float, f))] for c, f in (edits or [])]).encode()
        node = C.c_uint32()
        _check(lib().gtob_solver_lock_node(self._h, _ptr(st), len(steps), m, _ptr(fr), len(freqs or []), ej,
                                           label.encode(), C.byref(node)))
        return node.value

    def set_lock(self, node, sigma, label=""):
        s = np.ascontiguousarray(sigma, np.float32)
        _check(lib().gtob_solver_set_lock(self._h, int(node), _ptr(s), s.size, label.encode()))

    def clear_locks(self):
        _check(lib().gtob_solver_clear_locks(self._h))

    @property
    def num_locks(self):
        return lib().gtob_solver_num_locks(self._h)

    def path_view(self, path):
        """node_view's structure at the node `path` reaches (query.rs:353-461,
        490-640), host only: node, node_type, street, board, pot, put, player,
        actions (label, kind, amount), available_cards, locked, history."""
        st = np.array(_path_steps(path) + [0], np.int32)
        need = C.c_uint64()
        _check(lib().gtob_solver_path_view(self._h, _ptr(st), len(st) - 1, None, 0, C.byref(need)))
        buf = C.create_string_buffer(int(need.value))
        _check(lib().gtob_solver_path_view(self._h, _ptr(st), len(st) - 1, buf, need.value, C.byref(need)))
        return json.loads(buf.value.decode())

    def ensure_symmetric(self):
        _check(lib().gtob_solver_ensure_symmetric(self._h))

    def save(self, path):
        _check(lib().gtob_save(self._h, os.fspath(path).encode()))

    @staticmethod
    def load(path, storage="f32"):
        h = C.c_void_p()
        _check(lib().gtob_load(os.fspath(path).encode(), STORAGE[storage], C.byref(h)))
        # the loaded solver owns a spot rebuilt from the header; expose it too
        with open(path, "rb") as f:
            f.read(10)
            header = json.loads(f.readline())
        spot = Spot(header["config"], lenient=True)
        return Solver(spot, storage=storage, _handle=h)


def card_string(c):
    """cards.rs card_to_string: rank then suit ("Ah", "2c")."""
    return "23456789TJQKA"[c >> 2] + "cdhs"[c & 3]


def combo_string(c1, c2):
    """cards.rs:116-121 combo_to_string: the higher rank first, on equal ranks
    the higher suit first."""
    hi, lo = (c1, c2) if c1 > c2 else (c2, c1)
    a, b = (hi, lo) if (hi >> 2) >= (lo >> 2) else (lo, hi)
    return card_string(a) + card_string(b)


def _path_steps(path):
    """Path steps as the C ABI takes them: action indices, cards as -1 - card."""
    out = []
    for s in path:
        if isinstance(s, str):
            out.append(-1 - ("23456789TJQKA".index(s[0].upper()) * 4 + "cdhs".index(s[1].lower())))
        else:
            out.append(int(s))
    return out


class GpuSolver:
    """gpu/mod.rs GpuSolver: device buffers, CUDA-graph iterations, BR checks, syncs."""

    def __init__(self, solver, device_format=None, engine="staged"):
        """engine: "staged" (default: one CTA per node, its data staged in
        shared memory by bulk copies; showdowns batched by river board),
        "fused" (terminals evaluated inside their parents' kernels, f64
        terminal sums), "plain" (one launch per node kind and level, f64
        terminal sums), "fused32" (fused, f32 terminal sums) or "warp" (one
        warp per action node, fold children evaluated by that warp)."""
        h = C.c_void_p()
        eng = {"fused": 0, "plain": 1, "fused32": 2, "warp": 3, "staged": 4, "staged_river": 5}[engine]
        _check(lib().gtob_gpu_new_ex(solver._h, DEVICE_FORMAT[device_format], eng, C.byref(h)))
        self._h = h
        self.solver = solver

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.gtob_gpu_free(self._h)
            self._h = None

    def close(self):
        self.__del__()

    def iterate(self, n=1):
        _check(lib().gtob_gpu_iterate(self._h, int(n)))

    def iterate_profiled(self):
        p = Profile()
        _check(lib().gtob_gpu_iterate_profiled(self._h, C.byref(p)))
        return p

    def exploitability(self, solver=None):
        v = C.c_double()
        _check(lib().gtob_gpu_exploitability(self._h, (solver or self.solver)._h, C.byref(v)))
        return v.value

    def sync_to_cpu(self, solver=None):
        _check(lib().gtob_gpu_sync_to_cpu(self._h, (solver or self.solver)._h))

    def sync_strategy(self, solver=None):
        _check(lib().gtob_gpu_sync_strategy(self._h, (solver or self.solver)._h))

    def synchronize(self):
        _check(lib().gtob_gpu_synchronize(self._h))

    def update_locks(self, solver=None):
        _check(lib().gtob_gpu_update_locks(self._h, (solver or self.solver)._h))

    @property
    def iteration(self):
        return int(lib().gtob_gpu_iteration(self._h))

    def info(self):
        i = GpuInfo()
        _check(lib().gtob_gpu_info_get(self._h, C.byref(i)))
        return {k: (list(getattr(i, k)) if k in ("reach_slots", "device_action_nodes") else getattr(i, k))
                for k, _ in GpuInfo._fields_}

    def root_cfv(self, p, mode=0):
        out = np.zeros(self.solver.spot.nh[p], np.float32)
        _check(lib().gtob_gpu_root_cfv(self._h, int(p), int(mode), _ptr(out)))
        return out

    def export_arena(self, which, p):
        out = np.zeros(self.solver.spot.data_size[p], np.float32)
        _check(lib().gtob_gpu_export_arena(self._h, int(which), int(p), _ptr(out)))
        return out

    def read_node_static(self, which, node):
        """One action node's arena block through the allocation-free entry
        point (static device scratch of NODE_SCRATCH_ELEMS floats)."""
        t = self.solver.spot.tree()
        n = int(t["nchild"][node]) * self.solver.spot.nh[int(t["player"][node])]
        out = np.zeros(max(n, 1), np.float32)
        written = C.c_uint64()
        _check(lib().gtob_gpu_read_node_static(self._h, int(which), int(node), _ptr(out), out.size,
                                               C.byref(written)))
        return out[:written.value]

    def save(self, path, solver=None):
        """.gto written from the device arenas (config and locks from the host
        solver): the file sync_to_cpu + ensure_symmetric + Solver.save would
        give an f32 host solver, without a host arena copy."""
        _check(lib().gtob_gpu_save(self._h, (solver or self.solver)._h, os.fspath(path).encode()))

    @staticmethod
    def load(path, storage="f32", device_format=None, engine="staged"):
        """Solver.load + GpuSolver with the arenas streamed from the file into
        device memory.  Returns (solver, gpu); the host solver holds only the
        blocks the device does not, the rest after gpu.sync_to_cpu()."""
        sh, gh = C.c_void_p(), C.c_void_p()
        eng = {"fused": 0, "plain": 1, "fused32": 2, "warp": 3, "staged": 4, "staged_river": 5}[engine]
        _check(lib().gtob_gpu_load(os.fspath(path).encode(), STORAGE[storage], DEVICE_FORMAT[device_format], eng,
                                   C.byref(sh), C.byref(gh)))
        with open(path, "rb") as f:
            f.read(10)
            header = json.loads(f.readline())
        solver = Solver(Spot(header["config"], lenient=True), storage=storage, _handle=sh)
        gpu = GpuSolver.__new__(GpuSolver)
        gpu._h = gh
        gpu.solver = solver
        return solver, gpu

    def node_values(self, path, solver=None):
        """node_view's numbers (query.rs:490-600) at the node `path` reaches
        (ints: action indices, strings: cards), from device memory: dict with
        node, kind, player, reach/valid/ev per player and, at an action node,
        the actor's strategy and action_ev (num_actions x hands)."""
        sv = solver or self.solver
        steps = []
        for s in path:
            if isinstance(s, str):
                r, su = "23456789TJQKA".index(s[0].upper()), "cdhs".index(s[1].lower())
                steps.append(-1 - (r * 4 + su))
            else:
                steps.append(int(s))
        st = np.array(steps + [0], np.int32)
        sp = sv.spot
        nh = sp.nh
        reach = [np.zeros(nh[0], np.float32), np.zeros(nh[1], np.float32)]
        valid = [np.zeros(nh[0], np.float32), np.zeros(nh[1], np.float32)]
        eq = [np.zeros(nh[0], np.float32), np.zeros(nh[1], np.float32)]
        ev = [np.zeros(nh[0], np.float32), np.zeros(nh[1], np.float32)]
        mx = max(nh) * 64
        strat, aev = np.zeros(mx, np.float32), np.zeros(mx, np.float32)
        info = NodeInfo()
        _check(lib().gtob_gpu_node_values(self._h, sv._h, _ptr(st), len(steps), C.byref(info), _ptr(reach[0]),
                                          _ptr(reach[1]), _ptr(valid[0]), _ptr(valid[1]), _ptr(eq[0]), _ptr(eq[1]),
                                          _ptr(ev[0]), _ptr(ev[1]), _ptr(strat), _ptr(aev)))
        out = {"node": info.node, "kind": info.kind, "player": info.player, "reach": reach, "valid": valid,
               "eq": eq, "ev": ev}
        if info.kind == 0:
            na, h = info.num_actions, nh[info.player]
            out["strategy"] = strat[:na * h].reshape(na, h).copy()
            out["action_ev"] = aev[:na * h].reshape(na, h).copy()
        return out

    def node_view(self, path, solver=None):
        """query.rs node_view (490-640) at the node `path` reaches, its numbers
        from device memory (node_values) and its structure from the host
        (Solver.path_view): the reference's NodeView fields, with per player
        `hands` of combo, c1, c2, weight, reach, valid, eq, ev and, for the
        actor, strategy and evs (None where the reference has None)."""
        sv = solver or self.solver
        view = sv.path_view(path)
        vals = self.node_values(path, sv)
        sp = sv.spot

        def opt(x):
            x = float(x)
            return None if x != x else x
        players = []
        for p in (0, 1):
            c1, c2, w, _ = sp.hands(p)
            actor = view["node_type"] == "action" and view["player"] == p
            hands = []
            for i in range(sp.nh[p]):
                h = {"combo": combo_string(int(c1[i]), int(c2[i])), "c1": int(c1[i]), "c2": int(c2[i]),
                     "weight": float(w[i]), "reach": float(vals["reach"][p][i]), "valid": float(vals["valid"][p][i]),
                     "eq": opt(vals["eq"][p][i]), "ev": opt(vals["ev"][p][i])}
                if actor:
                    h["strategy"] = [float(x) for x in vals["strategy"][:, i]]
                    h["evs"] = [opt(x) for x in vals["action_ev"][:, i]]
                hands.append(h)
            players.append({"hands": hands})
        out = {k: view[k] for k in ("node_type", "street", "board", "pot", "put", "player", "actions",
                                    "available_cards")}
        out["players"] = players
        out["locked"] = view["locked"]
        out["history"] = view["history"]
        return out

    def exploit_view(self, path, exploiter, solver=None):
        """query.rs exploit_view (808-930): the ExploitView fields -- node_type,
        exploiter, player, actions, locked, per hand of the exploiter combo,
        c1, c2, weight, reach, valid, br_ev, cur_ev, gain and, where the
        exploiter acts, br_strategy and evs; avg_br_ev / avg_cur_ev / avg_gain
        -- numbers from device memory (exploit_values), structure from the host."""
        sv = solver or self.solver
        view = sv.path_view(path)
        vals = self.exploit_values(path, exploiter, sv)
        c1, c2, w, _ = sv.spot.hands(exploiter)

        def opt(x):
            x = float(x)
            return None if x != x else x
        actor = view["node_type"] == "action" and view["player"] == exploiter
        hands = []
        for i in range(sv.spot.nh[exploiter]):
            h = {"combo": combo_string(int(c1[i]), int(c2[i])), "c1": int(c1[i]), "c2": int(c2[i]),
                 "weight": float(w[i]), "reach": float(vals["reach"][i]), "valid": float(vals["valid"][i]),
                 "br_ev": opt(vals["br_ev"][i]), "cur_ev": opt(vals["cur_ev"][i]), "gain": opt(vals["gain"][i])}
            if actor:
                h["br_strategy"] = [float(x) for x in vals["br_strategy"][:, i]]
                h["evs"] = [opt(x) for x in vals["action_ev"][:, i]]
            hands.append(h)
        avg = [opt(x) for x in vals["averages"]]
        return {"node_type": view["node_type"], "exploiter": int(exploiter), "player": view["player"],
                "actions": view["actions"], "locked": view["locked"], "hands": hands,
                "avg_br_ev": avg[0], "avg_cur_ev": avg[1], "avg_gain": avg[2]}

    def runouts_report(self, path, solver=None):
        """query.rs runouts (964-1106) as its RunoutsReport: actions (of the
        action node after the first card, in descending card order, that
        leads to one), player, pot and per card (descending) the card string,
        freqs, eq and ev per player (None without mass)."""
        sv = solver or self.solver
        r = self.runouts(path, sv)

        def opt(x):
            x = float(x)
            return None if x != x else x
        actions = []
        for row in r["rows"]:
            v = sv.path_view(list(path) + [card_string(row["card"])])
            if v["node_type"] == "action":
                actions = v["actions"]
                break
        rows = [{"card": card_string(row["card"]), "freqs": [float(x) for x in row["freqs"]],
                 "eq": [opt(row["eq"][0]), opt(row["eq"][1])], "ev": [opt(row["ev"][0]), opt(row["ev"][1])]}
                for row in r["rows"]]
        return {"actions": actions, "player": r["player"] if r["player"] >= 0 else None, "pot": r["pot"],
                "rows": rows}

    def runouts(self, path, solver=None):
        """query.rs runouts at the chance node `path` reaches, from device
        memory: dict with player, pot and rows (card, freqs, eq, ev)."""
        sv = solver or self.solver
        st = np.array(_path_steps(path) + [0], np.int32)
        rows = (RunoutRow * 52)()
        freqs = np.zeros(52 * 64, np.float32)
        n, pl, na, pot = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        _check(lib().gtob_gpu_runouts(self._h, sv._h, _ptr(st), len(st) - 1, rows, _ptr(freqs), 52, 64, C.byref(n),
                                      C.byref(pl), C.byref(na), C.byref(pot)))
        out = []
        for k in range(n.value):
            r = rows[k]
            out.append({"card": r.card, "freqs": freqs[k * 64:k * 64 + na.value].copy(),
                        "eq": [r.eq[0], r.eq[1]], "ev": [r.ev[0], r.ev[1]]})
        return {"player": pl.value, "num_actions": na.value, "pot": pot.value, "rows": out}

    def exploit_values(self, path, exploiter, solver=None):
        """exploit_view's numbers (query.rs:808-930) for `exploiter` at the
        node `path` reaches, from device memory."""
        sv = solver or self.solver
        st = np.array(_path_steps(path) + [0], np.int32)
        nh = sv.spot.nh[exploiter]
        arrs = {k: np.zeros(nh, np.float32) for k in ("reach", "valid", "br_ev", "cur_ev", "gain")}
        strat, aev = np.zeros(nh * 64, np.float32), np.zeros(nh * 64, np.float32)
        avg = np.zeros(3, np.float32)
        info = NodeInfo()
        _check(lib().gtob_gpu_exploit_values(self._h, sv._h, _ptr(st), len(st) - 1, int(exploiter), C.byref(info),
                                             *[_ptr(arrs[k]) for k in ("reach", "valid", "br_ev", "cur_ev", "gain")],
                                             _ptr(strat), _ptr(aev), _ptr(avg)))
        out = dict(arrs, node=info.node, kind=info.kind, player=info.player, averages=avg)
        if info.kind == 0 and info.player == exploiter:
            na = info.num_actions
            out["br_strategy"] = strat[:na * nh].reshape(na, nh).copy()
            out["action_ev"] = aev[:na * nh].reshape(na, nh).copy()
        return out

    def discounts(self):
        out = np.zeros(3, np.float32)
        _check(lib().gtob_gpu_discounts(self._h, _ptr(out)))
        return out

    def time_iterations(self, n):
        """Run n iterations; return their device time in ms (CUDA events on the engine stream)."""
        ms = C.c_double()
        _check(lib().gtob_gpu_time_iterations(self._h, int(n), C.byref(ms)))
        return ms.value


ENGINES = {"fused": 0, "plain": 1, "fused32": 2, "warp": 3, "staged": 4, "staged_river": 5}


def nccl_unique_id():
    """ncclGetUniqueId for rank 0 to share with the other ranks (bytes)."""
    buf = (C.c_ubyte * 128)()
    _check(lib().gtob_nccl_unique_id(buf))
    return bytes(buf)


def sharded_gpu_solver(solver, rank, world, nccl_id, device_format=None, engine="staged"):
    """Shard `rank` of a spot split over `world` processes (one GPU each),
    its top chance values summed over NCCL; every rank calls this together."""
    buf = (C.c_ubyte * 128).from_buffer_copy(nccl_id)
    h = C.c_void_p()
    _check(lib().gtob_gpu_new_sharded(solver._h, DEVICE_FORMAT[device_format], ENGINES[engine], int(rank), int(world),
                                      buf, C.byref(h)))
    gpu = GpuSolver.__new__(GpuSolver)
    gpu._h = h
    gpu.solver = solver
    return gpu


def sharded_gpu_solver_host(solver, rank, world, reduce_fn, device_format=None, engine="staged"):
    """Shard `rank` of a spot split over `world` processes that sum over a
    channel of the caller's own: reduce_fn(values) gets a float32 array (the
    shard's values after a level of the up sweep) and must leave in it, in
    place, the element-wise sum over every rank -- for example
    torch.distributed.all_reduce on torch.from_numpy(values) in a gloo group.
    Every rank makes the same calls in the same order."""
    def tramp(user, ptr, count):
        try:
            reduce_fn(np.ctypeslib.as_array(ptr, shape=(int(count),)))
            return 0
        except BaseException:  # the error reaches the caller as a failed engine call
            import traceback
            traceback.print_exc()
            return 1
    cb = REDUCE_FN(tramp)
    h = C.c_void_p()
    _check(lib().gtob_gpu_new_sharded_host(solver._h, DEVICE_FORMAT[device_format], ENGINES[engine], int(rank),
                                           int(world), cb, None, C.byref(h)))
    gpu = GpuSolver.__new__(GpuSolver)
    gpu._h = h
    gpu.solver = solver
    gpu._reduce_cb = cb  # the C side keeps the pointer: keep the thunk alive with the engine
    return gpu


class Shards:
    """Every shard of one spot in this process on the current device, summing
    the split subtrees' values on the host: the sharded computation on one GPU."""

    def __init__(self, solver, nshards, device_format=None, engine="staged"):
        h = C.c_void_p()
        _check(lib().gtob_shards_new(solver._h, DEVICE_FORMAT[device_format], ENGINES[engine], int(nshards),
                                     C.byref(h)))
        self._h = h
        self.solver = solver

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.gtob_shards_free(self._h)
            self._h = None

    def iterate(self, n=1):
        _check(lib().gtob_shards_iterate(self._h, int(n)))

    def exploitability(self, solver=None):
        v = C.c_double()
        _check(lib().gtob_shards_exploitability(self._h, (solver or self.solver)._h, C.byref(v)))
        return v.value

    def export_arena(self, which, p):
        out = np.zeros(self.solver.spot.data_size[p], np.float32)
        _check(lib().gtob_shards_export_arena(self._h, int(which), int(p), _ptr(out)))
        return out

    def sync_to_cpu(self, solver=None, strategy_only=False):
        """Every shard's nodes into one host solver (GpuSolver.sync_to_cpu per shard)."""
        _check(lib().gtob_shards_sync_to_cpu(self._h, (solver or self.solver)._h, int(bool(strategy_only))))


BATCH_SEGMENT = np.dtype([("first", np.uint64), ("start", np.uint32), ("count", np.uint32), ("need", np.uint32),
                          ("spot", np.uint32), ("step", np.uint32), ("kind", np.int32), ("p", np.int32),
                          ("tile", np.int32)])


def batch_queue(spots, tile=4, use_iso=True):
    """The persistent batch kernel's work queue for these spots, built on the
    host (no GPU): (segments as a structured array, tickets, records)."""
    arr = (C.c_void_p * len(spots))(*[sp._h for sp in spots])
    n, nt, nr = C.c_int(), C.c_uint64(), C.c_uint64()
    _check(lib().gtob_spot_batch_queue(arr, len(spots), int(use_iso), int(tile), None, 0, C.byref(n), C.byref(nt),
                                       C.byref(nr)))
    out = np.zeros(n.value, BATCH_SEGMENT)
    _check(lib().gtob_spot_batch_queue(arr, len(spots), int(use_iso), int(tile), _ptr(out), n.value, C.byref(n),
                                       C.byref(nt), C.byref(nr)))
    return out, nt.value, nr.value


def shard_visited(spot, shard, nshards, use_iso=True):
    """Nodes shard `shard` of `nshards` visits (the plan partition, no GPU)."""
    out = np.zeros(spot.num_nodes, np.uint8)
    _check(lib().gtob_spot_shard_visited(spot._h, int(use_iso), int(shard), int(nshards), _ptr(out)))
    return out


class Batch:
    """Many spots solved on one GPU at once (the reference's batch report,
    solve_cli.rs:125-215, with the spots side by side): see gtob_batch_* in
    include/gtob.h."""

    def __init__(self, spots, storage="f32", algo="dcfr", use_iso=True, device_format=None, engine="staged",
                 keep_solvers=True):
        self.spots = list(spots)
        arr = (C.c_void_p * len(self.spots))(*[sp._h for sp in self.spots])
        eng = {"fused": 0, "plain": 1, "fused32": 2, "warp": 3, "staged": 4, "staged_river": 5}[engine]
        h = C.c_void_p()
        _check(lib().gtob_batch_new(arr, len(self.spots), STORAGE[storage], ALGO[algo], int(use_iso),
                                    DEVICE_FORMAT[device_format], eng, int(bool(keep_solvers)), C.byref(h)))
        self._h = h
        self.storage = storage

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.gtob_batch_free(self._h)
            self._h = None

    def run(self, max_iterations=300, target_pct=0.3, check_every=20, workers=8, persistent=False, window=16):
        """workers: spots in flight on their own engines and graphs; with
        persistent=True, `window` spots in flight whose iterations run as one
        persistent kernel launch each (gtob_batch_run_persistent)."""
        if persistent:
            _check(lib().gtob_batch_run_persistent(self._h, int(max_iterations), float(target_pct), int(check_every),
                                                   int(window)))
        else:
            _check(lib().gtob_batch_run(self._h, int(max_iterations), float(target_pct), int(check_every),
                                        int(workers)))

    def stats(self):
        """The last persistent run: launches, kernel_ms, tuned, tile, ctas_per_sm, grid."""
        st = BatchStats()
        _check(lib().gtob_batch_stats_get(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in BatchStats._fields_}

    def rows(self):
        out = []
        for i in range(len(self.spots)):
            r = BatchRow()
            _check(lib().gtob_batch_row_get(self._h, i, C.byref(r)))
            out.append({"status": r.status, "iterations": r.iterations, "exploit_pct": r.exploit_pct,
                        "seconds": r.seconds, "ev": [r.ev[0], r.ev[1]],
                        "error": lib().gtob_batch_error(self._h, i).decode(errors="replace")})
        return out

    def root_cfv(self, i, p):
        """Spot i's root counterfactual values (average strategies) per hand of p."""
        n = C.c_int()
        _check(lib().gtob_batch_root_cfv(self._h, int(i), int(p), None, 0, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        _check(lib().gtob_batch_root_cfv(self._h, int(i), int(p), _ptr(out), n.value, C.byref(n)))
        return out

    def solver(self, i):
        """The i-th host solver (owned by the batch, synced after run)."""
        h = lib().gtob_batch_solver(self._h, int(i))
        if not h:
            raise IndexError("no solver %d (out of range, or the batch keeps none)" % i)
        sv = Solver(self.spots[i], storage=self.storage, _handle=C.c_void_p(h))
        sv._owner = self
        return sv


def set_device(device):
    _check(lib().gtob_set_device(int(device)))


def gemm_bf16(a_bits, b_bits):
    """C = A B^T on the tcgen05 kernel: A (m x k) and B (n x k) as uint16 bf16
    bit patterns, C float32 (m, n multiples of 128, k of 64)."""
    a = np.ascontiguousarray(a_bits, np.uint16)
    b = np.ascontiguousarray(b_bits, np.uint16)
    m, k = a.shape
    n = b.shape[0]
    c = np.zeros((m, n), np.float32)
    _check(lib().gtob_gemm_bf16(_ptr(a), _ptr(b), m, n, k, _ptr(c)))
    return c


class LeafNet:
    """The turn-leaf value network: din -> nhidden x dh (GELU) -> dout, BF16
    weights and activations, FP32 accumulation, trained on the device."""

    def __init__(self, din, dh, nhidden, dout, seed=1):
        h = C.c_void_p()
        _check(lib().gtob_net_new(int(din), int(dh), int(nhidden), int(dout), int(seed), C.byref(h)))
        self._h = h
        self.din, self.dh, self.nhidden, self.dout = din, dh, nhidden, dout

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.gtob_net_free(self._h)
            self._h = None

    def _shape(self, layer):
        fin = self.din if layer == 0 else self.dh
        fout = self.dout if layer == self.nhidden else self.dh
        return fout, fin

    def params(self, layer):
        o, i = self._shape(layer)
        w = np.zeros((o, i), np.float32)
        b = np.zeros(o, np.float32)
        _check(lib().gtob_net_get_params(self._h, int(layer), _ptr(w), _ptr(b)))
        return w, b

    def set_params(self, layer, w, b):
        o, i = self._shape(layer)
        w = np.ascontiguousarray(w, np.float32).reshape(o, i)
        b = np.ascontiguousarray(b, np.float32).reshape(o)
        _check(lib().gtob_net_set_params(self._h, int(layer), _ptr(w), _ptr(b)))

    def grads(self, layer):
        o, i = self._shape(layer)
        w = np.zeros((o, i), np.float32)
        b = np.zeros(o, np.float32)
        _check(lib().gtob_net_get_grads(self._h, int(layer), _ptr(w), _ptr(b)))
        return w, b

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.din)
        y = np.zeros((x.shape[0], self.dout), np.float32)
        _check(lib().gtob_net_forward(self._h, _ptr(x), x.shape[0], _ptr(y)))
        return y

    def gradients(self, x, t, mask):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.din)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, self.dout)
        m = np.ascontiguousarray(mask, np.float32).reshape(-1, self.dout)
        loss = C.c_double()
        _check(lib().gtob_net_gradients(self._h, _ptr(x), _ptr(t), _ptr(m), x.shape[0], C.byref(loss)))
        return loss.value

    def train(self, x, t, mask, epochs, batch=1024, lr=1e-3, seed=1):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.din)
        t = np.ascontiguousarray(t, np.float32).reshape(-1, self.dout)
        m = np.ascontiguousarray(mask, np.float32).reshape(-1, self.dout)
        losses = np.zeros(epochs, np.float32)
        _check(lib().gtob_net_train(self._h, _ptr(x), _ptr(t), _ptr(m), x.shape[0], int(epochs), int(batch),
                                    C.c_float(lr), int(seed), _ptr(losses)))
        return losses


def dl_gpu_solver(solver, net, device_format=None, engine="staged"):
    """A depth-limited flop solve: the turn's betting chance nodes are leaves
    valued by `net` (a LeafNet of 2705 inputs and 2652 outputs)."""
    h = C.c_void_p()
    _check(lib().gtob_gpu_new_dl(solver._h, net._h, DEVICE_FORMAT[device_format], ENGINES[engine], C.byref(h)))
    gpu = GpuSolver.__new__(GpuSolver)
    gpu._h = h
    gpu.solver = solver
    gpu.net = net  # the solver holds the net too; keep the Python handle alive beside it
    return gpu


def dl_plan(spot):
    """The depth-limited plan of a flop spot, built on the host: (leaf nodes,
    pots, stacks, visited mask over the tree's nodes)."""
    n = C.c_int()
    _check(lib().gtob_spot_dl_plan(spot._h, None, None, None, 0, C.byref(n), None))
    nodes = np.zeros(n.value, np.uint32)
    pot = np.zeros(n.value, np.float32)
    stack = np.zeros(n.value, np.float32)
    vis = np.zeros(spot.num_nodes, np.uint8)
    _check(lib().gtob_spot_dl_plan(spot._h, _ptr(nodes), _ptr(pot), _ptr(stack), n.value, C.byref(n), _ptr(vis)))
    return nodes, pot, stack, vis


def dl_leaves(gpu):
    """(nodes, pots, stacks) of a depth-limited solver's leaves."""
    n = C.c_int()
    _check(lib().gtob_gpu_leaves(gpu._h, None, None, None, 0, C.byref(n)))
    nodes = np.zeros(n.value, np.uint32)
    pot = np.zeros(n.value, np.float32)
    stack = np.zeros(n.value, np.float32)
    _check(lib().gtob_gpu_leaves(gpu._h, _ptr(nodes), _ptr(pot), _ptr(stack), n.value, C.byref(n)))
    return nodes, pot, stack


def node_sweep(gpu, node, p, mode=1):
    """One evaluation sweep (mode 0 best response, 1 average strategies), then
    (node's value for p, reach of player 0, reach of player 1)."""
    nh = gpu.solver.spot.nh
    cfv = np.zeros(nh[p], np.float32)
    r0 = np.zeros(nh[0], np.float32)
    r1 = np.zeros(nh[1], np.float32)
    _check(lib().gtob_gpu_node_sweep(gpu._h, int(node), int(p), int(mode), _ptr(cfv), _ptr(r0), _ptr(r1)))
    return cfv, r0, r1


def node_strategy(gpu, node, num_actions, player):
    """The average strategy (num_actions x hands) of an action node on the device."""
    out = np.zeros(num_actions * gpu.solver.spot.nh[player], np.float32)
    _check(lib().gtob_gpu_node_strategy(gpu._h, int(node), _ptr(out)))
    return out.reshape(num_actions, -1)


def gemm_time_ms(m, n, k, reps=20):
    """Mean device ms of the tcgen05 product on m x k and n x k bf16 operands."""
    ms = C.c_double()
    _check(lib().gtob_gemm_time(int(m), int(n), int(k), int(reps), C.byref(ms)))
    return ms.value
