"""Regenerate tests/golden/reference_gpu_f32_dcfr.json from the reference's
own GPU run on its bench spot (bench/gpu_f32_dcfr.log: f32 arenas, DCFR,
exploitability every 10 iterations, RTX 3090).  The log's printed values are
the pins; nothing is computed here.  Usage:
    python tests/golden/make_reference_gpu_log.py /path/to/reference
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_reference_gpu_log.py <path of the reference project>")
    ref = sys.argv[1]
    path = os.path.join(ref, "bench", "gpu_f32_dcfr.log")
    pts = []
    with open(path) as f:
        for line in f:
            m = re.match(r"iter\s+(\d+)\s+exploitability\s+([\d.]+) chips \(([\d.]+)% pot\)", line)
            if m:
                pts.append({"iter": int(m.group(1)), "chips": float(m.group(2)), "pct_pot": float(m.group(3))})
    out = {"source": "bench/gpu_f32_dcfr.log", "spot": "bench_spot.json", "storage": "f32", "algo": "dcfr",
           "points": pts}
    with open(os.path.join(HERE, "reference_gpu_f32_dcfr.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(len(pts), "points")


if __name__ == "__main__":
    main()
