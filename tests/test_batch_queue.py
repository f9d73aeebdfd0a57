"""The persistent batch kernel's work queue, built on the host (no GPU):
the order its deadlock freedom rests on -- every ticket a segment waits for
belongs to its own spot's earlier steps and is numbered below the segment's
first ticket -- and coverage: one batched iteration visits every node record
exactly as often as the spot's own iteration does (each action node once in
the down sweep and once per up-sweep side, each chance edge, showdown batch
and chance node once per traverser, the discounts once, the root reach
twice), levels in the sweeps' order."""
import collections
import copy

import numpy as np
import pytest

import gtopen_b200 as g
from gtopen_b200 import workloads as W

DOWN, EDGE, SHOW, CHANCE, MINE, OPP = 2, 3, 4, 5, 6, 7


def _spots():
    a = W.small_flop_spot()
    b = W.iso_spot()
    c = copy.deepcopy(W.small_flop_spot())
    c["board"] = "KdQc4s"
    return [g.Spot(x) for x in (a, b, c, W.turn_spot(g.evaluate7, seed=2))]


@pytest.mark.parametrize("tile", [1, 4, 8])
def test_queue_order_and_coverage(tile):
    spots = _spots()
    seg, tickets, records = g.batch_queue(spots, tile=tile)
    nt = (seg["count"] + seg["tile"] - 1) // seg["tile"]
    assert np.all(seg["first"][1:] == seg["first"][:-1] + nt[:-1]) and seg["first"][0] == 0
    assert int(seg["first"][-1] + nt[-1]) == tickets and int(seg["count"].sum()) == records
    # ordered by step, then spot
    key = seg["step"].astype(np.int64) * len(spots) + seg["spot"]
    assert np.all(np.diff(key) >= 0)
    for s in range(len(spots)):
        mine = seg[seg["spot"] == s]
        mt = (mine["count"] + mine["tile"] - 1) // mine["tile"]
        for k in np.unique(mine["step"]):
            here = mine["step"] == k
            earlier = mine["step"] < k
            # a segment waits exactly for its spot's earlier steps ...
            assert np.all(mine["need"][here] == mt[earlier].sum())
            # ... whose tickets all come before its own first ticket
            if earlier.any():
                last = mine["first"][earlier] + mt[earlier]
                assert last.max() <= mine["first"][here].min()
        # coverage of one iteration
        cover = collections.defaultdict(collections.Counter)
        for r in mine:
            for i in range(int(r["start"]), int(r["start"] + r["count"])):
                cover[int(r["kind"])][i] += 1
        assert cover[0] == {0: 1} and cover[1] == {0: 2}
        n_act = max(cover[DOWN]) + 1
        for kind in (DOWN, MINE, OPP):
            assert set(cover[kind]) == set(range(n_act)) and set(cover[kind].values()) == {1}, kind
        for kind in (EDGE, SHOW, CHANCE):
            if cover[kind]:
                assert set(cover[kind]) == set(range(max(cover[kind]) + 1)), kind
                assert set(cover[kind].values()) == {2}, kind
        assert cover[SHOW], "no showdown batches"
        # each traverser's down sweep walks the levels down, the up sweep back up
        for p in (0, 1):
            half = mine[(mine["p"] == p) & np.isin(mine["kind"], [MINE, OPP])]
            assert np.all(np.diff(half["step"]) >= 0)
        downs = mine[mine["kind"] == DOWN]
        for part in np.split(downs, np.where(np.diff(downs["start"].astype(np.int64)) < 0)[0] + 1):
            assert np.all(np.diff(part["step"]) > 0)


def test_tile_changes_tickets_not_records():
    spots = _spots()[:2]
    a = g.batch_queue(spots, tile=1)
    b = g.batch_queue(spots, tile=8)
    assert a[2] == b[2] and a[1] > b[1]
