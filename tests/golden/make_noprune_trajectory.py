"""Regenerate tests/golden/bench_trajectory_noprune.json: the CPU oracle
WITHOUT zero-reach pruning -- the level-synchronous semantics the GPU engine
implements -- on the reference's bench_spot.json, exploitability every 10
iterations for 100 iterations, f32 and 16-bit arenas (DCFR).

"modes": terminal reach summed exactly (the GPU engine's order-independent
fixed-point sums, pyoracle exact=True); the GPU engine must land within 0.01%
of the pot of these values at every checkpoint.
"modes_f64": the same runs with the reference's f64 running sums (game.rs),
for comparison.
"pruned_exact": exact sums WITH the reference CPU engine's pruning, beside the
reference's own CPU logs (bench/new_f32_dcfr.log, new_i16_dcfr.log, kept in
bench_trajectory.json), which the f64 oracle reproduces to the printed digits:
how far the exact sums move the reference's own trajectory.
The reference's GPU run (bench/gpu_f32_dcfr.log, unpruned, f32 terminal sums
and a division in regret matching) is stored beside them.  Usage:
    python tests/golden/make_noprune_trajectory.py
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import pyoracle as po  # noqa: E402

MODES = {"f32_dcfr": False, "i16_dcfr": True}


def run(spot, comp, prune, exact, tag):
    sv = po.Solver(spot, compressed=comp, algo="dcfr", use_iso=True, prune=prune, exact=exact)
    vals = []
    t0 = time.time()
    for i in range(100):
        sv.iterate(1)
        if (i + 1) % 10 == 0:
            vals.append(sv.exploitability())
            print(tag, i + 1, vals[-1], "%.1fs" % (time.time() - t0), flush=True)
    return vals


def main():
    with open(os.path.join(HERE, "bench_spot.json")) as f:
        cfg = json.load(f)
    with open(os.path.join(HERE, "reference_gpu_f32_dcfr.json")) as f:
        ref_gpu = [p["chips"] for p in json.load(f)["points"]]
    spot = po.Spot(cfg)
    out = {"spot": "bench_spot.json", "pot": cfg["tree"]["starting_pot"], "iters": list(range(10, 101, 10)),
           "modes": {}, "modes_f64": {}, "pruned_exact": {}, "reference_gpu_f32_dcfr": ref_gpu}
    for mode, comp in MODES.items():
        out["modes"][mode] = run(spot, comp, False, True, "exact " + mode)
        out["modes_f64"][mode] = run(spot, comp, False, False, "f64 " + mode)
        out["pruned_exact"][mode] = run(spot, comp, True, True, "pruned exact " + mode)
    with open(os.path.join(HERE, "bench_trajectory_noprune.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
