"""The allocation-free entry point gtob_gpu_read_node_static against the
existing gtob_gpu_export_arena: the same node block, bit for bit, on two
calls in a row (the static scratch is reused by the second call), for f32,
16-bit and FP8 arenas and for PCFR+'s predictions; and a block larger than
the static scratch is refused.
Collected last on purpose: it must pass alone and after every other test.
"""
import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _slice(arena, spot, node):
    t = spot.tree()
    off = int(t["data_off"][node])
    n = int(t["nchild"][node]) * spot.nh[int(t["player"][node])]
    return arena[off:off + n]


def _two_nodes(spot):
    """The root (OOP) and the first IP action node."""
    t = spot.tree()
    ip = np.nonzero((t["kind"] == 0) & (t["player"] == 1))[0]
    return 0, int(ip[0])


@pytest.mark.parametrize("storage,device_format,algo", [("f32", None, "dcfr"), ("compressed", None, "dcfr"),
                                                      ("f32", "fp8", "dcfr"), ("f32", None, "pcfr+"),
                                                      ("compressed", None, "pcfr+")])
def test_static_read_equals_export_two_calls_in_a_row(storage, device_format, algo):
    spot = g.Spot(W.small_flop_spot())
    host = g.Solver(spot, storage=storage, algo=algo, use_iso=False)
    gpu = g.GpuSolver(host, device_format=device_format)
    gpu.iterate(7)
    a, b = _two_nodes(spot)
    kinds = (0, 1, 2) if algo == "pcfr+" else (0, 1)  # regrets, strategy sums, predictions
    for rnd in range(2):
        for which in kinds:
            # two calls in a row through the static scratch ...
            ra = gpu.read_node_static(which, a)
            sb = gpu.read_node_static(which, b)
            # ... against the existing allocating entry point
            ea = _slice(gpu.export_arena(which, 0), spot, a)
            eb = _slice(gpu.export_arena(which, 1), spot, b)
            assert ra.shape == ea.shape and sb.shape == eb.shape
            assert np.array_equal(ra, ea), (storage, device_format, which, rnd, float(np.abs(ra - ea).max()))
            assert np.array_equal(sb, eb), (storage, device_format, which, rnd, float(np.abs(sb - eb).max()))
            assert np.any(ra != 0.0) and np.any(sb != 0.0)
        gpu.iterate(3)


def test_static_read_refuses_blocks_beyond_the_scratch():
    cfg = W.river_spot()
    # 15 bet sizes + all-in + check at the root: 17 actions x 1081 hands > 16384
    cfg["tree"] = W.tree_config(100, 400, tuple(str(5 * k) for k in range(1, 16)) + ("a",), ("2.5x",), 1)
    spot = g.Spot(cfg)
    t = spot.tree()
    na_root = int(t["nchild"][0])
    assert na_root * spot.nh[0] > g.NODE_SCRATCH_ELEMS
    host = g.Solver(spot, use_iso=False)
    gpu = g.GpuSolver(host)
    gpu.iterate(2)
    with pytest.raises(g.GtobError) as e:
        gpu.read_node_static(0, 0)
    assert "static scratch" in str(e.value)
    # a smaller node of the same spot still reads: IP facing the smallest bet
    small = int(spot.children()[int(t["child_start"][0]) + 1])
    assert int(t["kind"][small]) == 0 and int(t["nchild"][small]) * spot.nh[1] <= g.NODE_SCRATCH_ELEMS
    r = gpu.read_node_static(1, small)
    assert np.array_equal(r, _slice(gpu.export_arena(1, 1), spot, small))
