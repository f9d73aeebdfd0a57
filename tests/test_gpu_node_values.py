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


def _expected_exploit(ospot, osv, tree, path, p):
    """exploit_view's numbers (query.rs:808-930) from the oracle's best-response
    and average traversals (no iso: the browsed branch is the canonical one)."""
    steps = _steps(path)
    node, br_node, br_child, r0, r1 = osv.node_values(steps, p, avg=False)
    _, cur, _, _, _ = osv.node_values(steps, p, avg=True)
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
    actor = tree["kind"][node] == 0 and tree["player"][node] == p
    ok = valid > 1e-9
    out = {"node": node, "reach": reach[p], "valid": valid}
    if actor:
        na = int(tree["nchild"][node])
        acfv = br_child[:na]
        br = acfv.max(0)
        m = br
        eps = np.maximum(np.abs(m) * np.float32(1e-5), np.float32(1e-5))
        win = (m[None, :] - acfv) <= eps[None, :]
        w = np.maximum(win.sum(0), 1).astype(np.float32)
        out["br_strategy"] = np.where(win, np.float32(1.0) / w, np.float32(0.0))
        aev = np.full(acfv.shape, np.nan)
        aev[:, ok] = acfv[:, ok] / valid[ok] + put
        out["action_ev"] = aev
    else:
        br = br_node
    be, ce = np.full(len(valid), np.nan), np.full(len(valid), np.nan)
    be[ok] = br[ok] / valid[ok] + put
    ce[ok] = cur[ok] / valid[ok] + put
    out["br_ev"], out["cur_ev"] = be, ce
    return out


@pytest.mark.parametrize("device_format", ["f32", "i16"])
def test_exploit_values_match_oracle(device_format):
    cfg = W.small_flop_spot()
    exact = device_format == "f32"
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32" if exact else "compressed", use_iso=False)
    gpu = g.GpuSolver(host, device_format=device_format)
    gpu.iterate(25)
    paths = [[], [0], [1], [1, 0], [1, 1], [0, 0, "Ah"], [0, 1, 1, "5d", 0]]
    got = {(tuple(pa), p): gpu.exploit_values(pa, p, host) for pa in paths for p in (0, 1)}
    gpu.sync_to_cpu(host)
    ospot = po.Spot(cfg)
    osv = po.Solver(ospot, compressed=False, use_iso=False, prune=False)
    for which in (0, 1):
        for q in (0, 1):
            osv.set_arena(which, q, host.arena(which, q))
    tree = spot.tree()
    for (pa, p), v in got.items():
        exp = _expected_exploit(ospot, osv, tree, list(pa), p)
        assert v["node"] == exp["node"], pa
        if exact:
            assert np.array_equal(v["reach"], exp["reach"]), pa
        _close(v["reach"], exp["reach"], ("reach", pa, p))
        _close(v["valid"], exp["valid"].astype(np.float32), ("valid", pa, p))
        _close(v["br_ev"], exp["br_ev"], ("br_ev", pa, p))
        _close(v["cur_ev"], exp["cur_ev"], ("cur_ev", pa, p))
        assert (np.nan_to_num(v["gain"], nan=0.0) >= -1e-3).all(), (pa, p)  # a best response never loses
        if "action_ev" in exp:
            _close(v["action_ev"], exp["action_ev"], ("action_ev", pa, p))
            # ties can split differently when values agree only to the bar
            agree = (v["br_strategy"] == exp["br_strategy"]).all(0)
            assert agree.mean() > 0.99, (pa, p)
        w = v["reach"].astype(np.float64) * v["valid"].astype(np.float64)
        m = ~np.isnan(v["br_ev"]) & (w > 0)
        if w[m].sum() > 1e-12:
            assert abs(v["averages"][0] - (w[m] * v["br_ev"][m]).sum() / w[m].sum()) < 1e-3
            assert abs(v["averages"][2] - (v["averages"][0] - v["averages"][1])) < 1e-3


def test_exploit_values_mirror_branch():
    """KsQs2d: the club branch is the heart branch's mirror; the browsed
    hands read the representative's values through the suit swap."""
    cfg = W.iso_spot()
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", use_iso=True)
    gpu = g.GpuSolver(host)
    gpu.iterate(15)
    a = gpu.exploit_values([0, 0, "Ac"], 0, host)
    b = gpu.exploit_values([0, 0, "Ah"], 0, host)
    assert a["node"] == b["node"]
    c1, c2, _, _ = spot.hands(0)
    swap = {0: 2, 2: 0, 1: 1, 3: 3}
    idx = {(int(x), int(y)): i for i, (x, y) in enumerate(zip(c1, c2))}
    for i, (x, y) in enumerate(zip(c1, c2)):
        xs, ys = (int(x) & ~3) | swap[int(x) & 3], (int(y) & ~3) | swap[int(y) & 3]
        j = idx[(max(xs, ys), min(xs, ys))]
        for k in ("br_ev", "cur_ev", "reach", "valid"):
            va, vb = a[k][i], b[k][j]
            assert (np.isnan(va) and np.isnan(vb)) or va == vb, (k, i, j, va, vb)
