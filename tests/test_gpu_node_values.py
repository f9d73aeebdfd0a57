"""Node queries over the device arenas (gtob_gpu_node_values) against the
oracle's node_view traversals (query.rs:304-340 walk_path, best_response.rs
avg_into) on the same strategies: the GPU solve is synced to an f32 host
solver, symmetrised, and handed to the oracle.  Reach along the path is
bit-exact; values within 1e-5 relative + 1e-3 chips (f32 sums in another
order, f64 showdown sums grouped differently)."""
import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _steps(path):
    out = []
    for s in path:
        if isinstance(s, str):
            out.append(-1 - ("23456789TJQKA".index(s[0].upper()) * 4 + "cdhs".index(s[1].lower())))
        else:
            out.append(int(s))
    return out


def _expected(ospot, osv, tree, path):
    """node_view's numbers (query.rs:490-600) from the oracle's traversals."""
    steps = _steps(path)
    res = {}
    for p in (0, 1):
        node, cfv, child, r0, r1 = osv.node_values(steps, p)
        reach = (r0, r1)
        ro = reach[1 - p].astype(np.float64)
        oc1, oc2, _ = ospot.hands(1 - p)
        c1, c2, _ = ospot.hands(p)
        same = ospot.same_combo(p)
        s = np.zeros(52)
        np.add.at(s, oc1, ro)
        np.add.at(s, oc2, ro)
        same_r = np.where(same != 0xFFFFFFFF, ro[np.minimum(same, len(ro) - 1)], 0.0)
        valid = ro.sum() - s[c1] - s[c2] + same_r
        put = tree["put0" if p == 0 else "put1"][node]
        ok = valid > 1e-9
        actor = tree["kind"][node] == 0 and tree["player"][node] == p
        ev = np.full(len(valid), np.nan)
        if actor:
            na = int(tree["nchild"][node])
            sig = osv.avg_strategy(node, na, len(valid)).reshape(na, -1).astype(np.float64)
            aev = np.full((na, len(valid)), np.nan)
            aev[:, ok] = child[:na, ok] / valid[ok] + put
            ev[ok] = (sig[:, ok] * aev[:, ok]).sum(0)
            res["strategy"], res["action_ev"] = sig, aev
        else:
            ev[ok] = cfv[ok] / valid[ok] + put
        res[p] = (node, reach, valid, ev)
    return res


def _close(a, b, what):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    assert np.array_equal(np.isnan(a), np.isnan(b)), what
    m = ~np.isnan(a)
    err = np.abs(a[m] - b[m]) - (1e-3 + 1e-5 * np.abs(b[m]))
    assert (err <= 0).all(), (what, float(np.abs(a[m] - b[m]).max()))


def _check(cfg, use_iso, device_format, paths):
    """f32 arenas: reach and strategies bit-exact against the oracle.  16-bit
    arenas: the strategies follow the quant rule (cfr.rs:712-722), exact
    against the synced compressed host solver; the oracle then runs the f32
    rule on the decoded values, so reach and values get the value bar."""
    exact = device_format == "f32"
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32" if exact else "compressed", use_iso=use_iso)
    gpu = g.GpuSolver(host, device_format=device_format)
    gpu.iterate(25)
    got = {tuple(p): gpu.node_values(p, host) for p in paths}
    gpu.sync_to_cpu(host)
    host.ensure_symmetric()
    ospot = po.Spot(cfg)
    osv = po.Solver(ospot, compressed=False, use_iso=use_iso, prune=False)
    for which in (0, 1):
        for p in (0, 1):
            osv.set_arena(which, p, host.arena(which, p))
    tree = spot.tree()
    for path in paths:
        v = got[tuple(path)]
        exp = _expected(ospot, osv, tree, path)
        for p in (0, 1):
            node, reach, valid, ev = exp[p]
            assert v["node"] == node, path
            if exact:
                assert np.array_equal(v["reach"][0], reach[0]) and np.array_equal(v["reach"][1], reach[1]), path
            else:
                _close(v["reach"][0], reach[0], ("reach0", path))
                _close(v["reach"][1], reach[1], ("reach1", path))
            _close(v["valid"][p], valid.astype(np.float32), ("valid", path, p))
            _close(v["ev"][p], ev, ("ev", path, p))
        if v["kind"] == 0:
            if exact:
                assert np.array_equal(v["strategy"], exp["strategy"].astype(np.float32)), path
            else:
                assert np.array_equal(v["strategy"].ravel(), host.average_strategy(v["node"]).ravel()), path
            _close(v["action_ev"], exp["action_ev"], ("action_ev", path))


@pytest.mark.parametrize("device_format", ["f32", "i16"])
def test_node_values_match_oracle(device_format):
    paths = [[], [0], [1], [0, 0], [1, 0], [1, 1], [0, 0, "Ah"], [0, 0, "Ah", 0], [0, 1, 1, "5d", 0, 0, "3s"]]
    _check(W.small_flop_spot(), False, device_format, paths)


def test_node_values_through_symmetric_branches():
    """iso spot KsQs2d: hearts and clubs mirror each other; the club branch is
    read from the heart branch the device holds."""
    paths = [[0, 0, "Ah"], [0, 0, "Ac"], [0, 0, "Ac", 1], [0, 0, "Ac", 0, 0, "3h"]]
    _check(W.iso_spot(), True, "f32", paths)
