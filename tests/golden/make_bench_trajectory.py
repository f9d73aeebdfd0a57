"""Regenerate tests/golden/bench_trajectory.json: the CPU oracle (prune on,
the reference CPU engine's semantics) run on the reference's bench_spot.json
for 100 iterations, exploitability every 10, in the three modes the
reference's bench logs record (bench/new_f32_dcfr.log, new_i16_dcfr.log,
new_i16_pcfr.log).  The reference values are stored beside ours so the
committed file is self-checking.  Usage:
    python tests/golden/make_bench_trajectory.py [--iters 100]
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import pyoracle as po  # noqa: E402

# Printed values of the reference's own logs (chips at iterations 10..100).
REFERENCE = {
    "f32_dcfr": [33.7904, 9.3381, 4.8733, 3.3154, 2.3677, 1.7728, 1.3505, 1.0533, 0.8316, 0.6747],
    "i16_dcfr": [33.5076, 9.2809, 4.8721, 3.3099, 2.3737, 1.7740, 1.3562, 1.0590, 0.8350, 0.6787],
    "i16_pcfr": [27.4101, 9.7649, 5.9891, 4.3956, 3.6676, 3.1206, 2.6582, 2.3066, 2.0422, 1.8363],
}
MODES = {"f32_dcfr": (False, "dcfr"), "i16_dcfr": (True, "dcfr"), "i16_pcfr": (True, "pcfr+")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--modes", default=",".join(MODES))
    a = ap.parse_args()
    cfg = json.load(open(os.path.join(HERE, "bench_spot.json")))
    spot = po.Spot(cfg)
    out = {"spot": "bench_spot.json", "nodes": spot.num_nodes, "hands": spot.nh, "modes": {}}
    for mode in a.modes.split(","):
        comp, algo = MODES[mode]
        sv = po.Solver(spot, compressed=comp, algo=algo, use_iso=True, prune=True)
        ours = []
        t0 = time.time()
        for i in range(a.iters):
            sv.iterate(1)
            if (i + 1) % 10 == 0:
                ours.append(round(sv.exploitability(), 4))
                print(mode, i + 1, ours[-1], "%.1fs" % (time.time() - t0), flush=True)
        out["modes"][mode] = {"oracle": ours, "reference": REFERENCE[mode][: len(ours)]}
    with open(os.path.join(HERE, "bench_trajectory.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
