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
    osv = po.Solver(ospot, compressed=False, use_iso=use_iso, prune=False, exact=True)
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
    osv = po.Solver(ospot, compressed=False, use_iso=False, prune=False, exact=True)
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


def _equity(ospot, p, ro, dealt, board):
    """best_response.rs:292-386 / game.rs:580-653 restated over the oracle's
    river tables (the test's own reference for the equity numbers)."""
    oc1, oc2, _ = ospot.hands(1 - p)
    c1, c2, _ = ospot.hands(p)
    same = ospot.same_combo(p)
    nh = len(c1)
    win, tie, valid = np.zeros(nh), np.zeros(nh), np.zeros(nh)

    def sweep(d, r):
        ms, mi = ospot.river(p, d)
        os_, oi = ospot.river(1 - p, d)
        r = r.astype(np.float64)
        t_all = r[oi].sum()
        s_all = np.zeros(52)
        np.add.at(s_all, oc1[oi], r[oi])
        np.add.at(s_all, oc2[oi], r[oi])
        j, t, s = 0, 0.0, np.zeros(52)
        lower = np.zeros(len(mi))
        for k in range(len(mi)):
            while j < len(oi) and os_[j] < ms[k]:
                x = oi[j]
                t += r[x]
                s[oc1[x]] += r[x]
                s[oc2[x]] += r[x]
                j += 1
            lower[k] = t - s[c1[mi[k]]] - s[c2[mi[k]]]
        j, t, s = len(oi), 0.0, np.zeros(52)
        for k in range(len(mi) - 1, -1, -1):
            while j > 0 and os_[j - 1] > ms[k]:
                j -= 1
                x = oi[j]
                t += r[x]
                s[oc1[x]] += r[x]
                s[oc2[x]] += r[x]
            i = mi[k]
            higher = t - s[c1[i]] - s[c2[i]]
            sr = r[same[i]] if same[i] != 0xFFFFFFFF else 0.0
            v = t_all - s_all[c1[i]] - s_all[c2[i]] + sr
            win[i] += lower[k]
            tie[i] += v - lower[k] - higher
            valid[i] += v

    omask = lambda c: (oc1 == c) | (oc2 == c)
    nb = len(dealt) + 3
    if nb == 5:
        sweep(list(dealt), ro)
    else:
        bd = set(board)
        free = [c for c in range(52) if c not in bd and c not in dealt]
        if nb == 4:
            for c in free:
                sweep(list(dealt) + [c], np.where(omask(c), 0.0, ro))
        else:
            for a in range(len(free)):
                for b in range(a + 1, len(free)):
                    ta, tb = free[a], free[b]
                    sweep([ta, tb], np.where(omask(ta) | omask(tb), 0.0, ro))
    out = np.full(nh, np.nan)
    ok = valid > 1e-12
    out[ok] = (win[ok] + 0.5 * tie[ok]) / valid[ok]
    return out


def test_equity_and_runouts_match_oracle():
    cfg = W.small_flop_spot()
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", use_iso=False)
    gpu = g.GpuSolver(host)
    gpu.iterate(20)
    nv = gpu.node_values([1, 1, "Ah"], host)
    ro_turn = gpu.runouts([0, 0], host)
    ro_river = gpu.runouts([0, 0, "Ah", 0, 0], host)
    gpu.sync_to_cpu(host)
    ospot = po.Spot(cfg)
    osv = po.Solver(ospot, compressed=False, use_iso=False, prune=False, exact=True)
    for which in (0, 1):
        for q in (0, 1):
            osv.set_arena(which, q, host.arena(which, q))
    card = lambda s: "23456789TJQKA".index(s[0]) * 4 + "cdhs".index(s[1])
    board = [card(cfg["board"][i:i + 2]) for i in range(0, len(cfg["board"]), 2)]
    # equity at a turn node (river runouts enumerated)
    for p in (0, 1):
        _, _, _, r0, r1 = osv.node_values(_steps([1, 1, "Ah"]), p)
        ro = (r0, r1)[1 - p]
        _close(nv["eq"][p], _equity(ospot, p, ro, [card("Ah")], board), ("eq", p))
    tree = spot.tree()
    for path, rep in (([0, 0], ro_turn), ([0, 0, "Ah", 0, 0], ro_river)):
        dealt = [card(s) for s in path if isinstance(s, str)]
        assert len(rep["rows"]) > 0
        assert [r["card"] for r in rep["rows"]] == sorted([r["card"] for r in rep["rows"]], reverse=True)
        for row in rep["rows"]:
            c = row["card"]
            cp = path + ["23456789TJQKA"[c >> 2] + "cdhs"[c & 3]]
            for p in (0, 1):
                node, cfv, _, r0, r1 = osv.node_values(_steps(cp), p)
                reach = (r0, r1)
                ro = reach[1 - p].astype(np.float64)
                oc1, oc2, _ = ospot.hands(1 - p)
                c1, c2, _ = ospot.hands(p)
                same = ospot.same_combo(p)
                s = np.zeros(52)
                np.add.at(s, oc1, ro)
                np.add.at(s, oc2, ro)
                valid = ro.sum() - s[c1] - s[c2] + np.where(same != 0xFFFFFFFF, ro[np.minimum(same, len(ro) - 1)], 0.0)
                rp = reach[p].astype(np.float64)
                eq = _equity(ospot, p, reach[1 - p], dealt + [c], board)
                m = ~np.isnan(eq)
                w = rp[m] * valid[m]
                exp_eq = (w * eq[m]).sum() / w.sum() if w.sum() > 1e-12 else np.nan
                put = tree["put0" if p == 0 else "put1"][node]
                ok = (valid > 1e-9) & (rp > 0)
                w = rp[ok] * valid[ok]
                exp_ev = (w * (cfv[ok] / valid[ok] + put)).sum() / w.sum() if w.sum() > 1e-12 else np.nan
                _close([row["eq"][p]], [exp_eq], ("runout eq", path, c, p))
                _close([row["ev"][p]], [exp_ev], ("runout ev", path, c, p))
            if tree["kind"][node] == 0:
                pl = int(tree["player"][node])
                na = int(tree["nchild"][node])
                _, _, _, r0, r1 = osv.node_values(_steps(cp), pl)
                rp = (r0, r1)[pl].astype(np.float64)
                sig = osv.avg_strategy(node, na, len(rp)).reshape(na, -1).astype(np.float64)
                exp_f = (sig * rp[None, :]).sum(1) / rp.sum()
                assert rep["player"] == pl and rep["num_actions"] == na
                assert np.allclose(row["freqs"], exp_f, rtol=1e-5, atol=1e-6), (path, c)
