#!/usr/bin/env python
"""Benchmark of the GTOpen postflop discounted-CFR iteration on B200.

A step is one DCFR iteration (both traversals, alternating updates) of one
spot.  Default workload: the flop single-raised-pot configuration (3-card
board, OOP top 40% / IP top 55% of combos, pot 55, stack 975, bets
{33,75,a}, raises {2.5x,a}, 3 raises: 10,835,022 nodes, 470 x 647 hands)
with i16/u16 arenas, inputs synthesised from a fixed seed.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

value     = iterations/s over all ranks (each rank solves its own replica;
            weak scaling, no data-path collective), device time from CUDA
            events on the engine's stream, max over ranks.
e2e       = the same metric through the C ABI from host arenas: upload
            (GpuSolver::new), K iterations, one exploitability check, and the
            arena download (sync_to_cpu), wall clock.
roofline  = algorithmic bytes per iteration / device time per iteration vs
            the measured HBM copy bandwidth.
cpu_baseline / --impl reference = the CPU oracle (the reference CPU engine's
            algorithm, restated in C++ and run with OpenMP over chance
            branches) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAK_FALLBACK = 6650.0


def load_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return PEAK_FALLBACK, "fallback"


def make_config(name, evaluate7=None):
    """The workload's spot config.  evaluate7 draws the strength-shaped ranges:
    the product's evaluator by default; the reference arm passes the oracle's
    (bit-identical, pinned to the reference's evaluator tests) so that its
    process never loads the product library."""
    from gtopen_b200 import workloads as W
    if evaluate7 is None:
        import gtopen_b200 as g
        evaluate7 = g.evaluate7
    if name == "flop":
        return W.flop_spot(evaluate7, seed=3)
    if name == "flop_narrow":  # the flop's board and ranges on a narrow tree (profiling case)
        return W.flop_spot(evaluate7, seed=3, bet=("75", "a"), raise_=("a",), max_raises=2)
    if name == "turn":
        return W.turn_spot(evaluate7, seed=2)
    if name == "river":
        return W.river_spot(seed=1)
    if name == "bench_spot":
        with open(os.path.join(ROOT, "tests", "golden", "bench_spot.json")) as f:
            return json.load(f)
    raise SystemExit("unknown workload " + name)


class Clocks:
    """nvidia-smi samples during the timed region (median SM clock, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus, backend=None):
    """One process per GPU (torchrun env).  NCCL on GPUs; gloo when no GPU is
    visible (the multi-rank plumbing's CPU tests).  A short process-group
    timeout makes ranks that wait on a missing peer fail instead of hanging."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        timeout = datetime.timedelta(seconds=120)
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=timeout)
    return world, rank, local


def allmax(x, world):
    """Max over ranks (device times are reported as the slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --storage: compressed = i16/u16 host and device arenas (the reference CLI
# default); f32; fp8 = f32 host arenas, FP8 E4M3 device arenas (precision study)
# DRAM bytes (read + write) of one CFR iteration, summed over every launch of
# an iteration in a one-pass ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum).  flop_narrow is captured directly (6.690 GB per
# iteration, profiles/staged_engine_flop_narrow_launches.md); the flop's figure
# is that capture scaled by the ratio of algorithmic bytes (127.48 / 3.946 GB).
# Only for the configurations captured.
MEASURED_TRAFFIC = {("flop_narrow", "i16sr", "staged"): 6.690e9, ("flop", "i16sr", "staged"): 216.1e9}

# i16sr = i16/u16 arenas whose update requantises with stochastic rounding
# (the default: store.rs's round-to-nearest stalls on the flop workload)
HOST_STORAGE = {"compressed": "compressed", "i16sr": "compressed", "f32": "f32", "fp8": "f32"}
DEVICE_FORMAT = {"compressed": None, "i16sr": "i16sr", "f32": None, "fp8": "fp8"}
DTYPE = {"compressed": "i16", "i16sr": "i16", "f32": "f32", "fp8": "fp8_e4m3"}
ARENA_DESC = {"compressed": "i16/u16 per-node scale, round to nearest (store.rs)",
              "i16sr": "i16/u16 per-node scale, stochastic rounding", "f32": "f32",
              "fp8": "FP8 E4M3 per-node scale"}
HOST_BYTES = {"compressed": 2, "i16sr": 2, "f32": 4, "fp8": 4}


def host_cpus():
    """(physical cores, logical CPUs, model name) of the CPUs this process may
    run on (its affinity mask; /proc/cpuinfo's physical id / core id pairs)."""
    try:
        allowed = os.sched_getaffinity(0)
    except (AttributeError, OSError):
        allowed = set(range(os.cpu_count() or 1))
    cores, model, cpu = set(), "", None
    phys = core = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f.read().splitlines() + [""]:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "processor":
                    cpu = int(v)
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif k == "model name" and not model:
                    model = v
                elif not line.strip():
                    if cpu is not None and cpu in allowed:
                        cores.add((phys, core) if core is not None else ("cpu", cpu))
                    cpu = phys = core = None
    except OSError:
        pass
    return max(1, len(cores) or len(allowed)), len(allowed), model


def cpu_baseline(cfg, storage, steps, threads=None):
    """The oracle (reference CPU engine restated, pruning on) on the host
    cores: one thread per physical core unless told otherwise, the reference
    CLI's default (SOLVER_THREADS, README.md: SMT hurts this workload)."""
    from oracle import pyoracle as po
    phys, logical, _ = host_cpus()
    n = threads or phys
    po.set_threads(n)
    t0 = time.perf_counter()
    spot = po.Spot(cfg)
    build_s = time.perf_counter() - t0
    sv = po.Solver(spot, compressed=storage in ("compressed", "i16sr"), fp8=storage == "fp8", algo="dcfr",
                   use_iso=True, prune=True, stochastic=storage == "i16sr")
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        sv.iterate(1)
        times.append(time.perf_counter() - t)
    return {"iter_s": times, "build_s": build_s, "cores": n, "physical_cores": phys, "logical_cpus": logical,
            "cpu_model": host_cpus()[2]}


def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import pyoracle as po
    cfg = make_config(args.workload, evaluate7=po.evaluate7)
    k = max(1, args.steps)
    w = max(0, args.warmup)
    r = cpu_baseline(cfg, args.storage, k + w, args.cpu_threads)
    timed = r["iter_s"][w:]
    total = sum(timed)
    value = len(timed) / total
    line = {
        "impl": "reference", "metric": "CFR iterations/s (time-to-0.3%-pot exploitability & HBM GB/s vs peak)",
        "value": value, "unit": "iter/s", "n_gpus": args.gpus, "steps": len(timed), "warmup": w,
        "ms_per_step": 1000.0 * total / len(timed), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPE[args.storage], "data": "synthetic (seeded spot)",
        "config": workload_config(args, cfg),
        "cpu_baseline": {"value": value, "unit": "iter/s", "cores": r["cores"], "kind": "port",
                         "cpu_model": r["cpu_model"], "physical_cores": r["physical_cores"],
                         "logical_cpus": r["logical_cpus"],
                         "sample": "%d full DCFR iterations of the workload on the CPU oracle "
                                   "(reference cfr.rs semantics, pruning on, OpenMP over chance cards)" % len(timed)},
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(args, cfg):
    return {"workload": {"flop": "flop SRP: 3-card board seed 3, OOP top40%/IP top55%, pot 55 stack 975, "
                                 "bets {33,75,a} raises {2.5x,a} max 3 raises",
                         "flop_narrow": "flop SRP board and ranges (seed 3, 470 v 647) on a narrow tree: "
                                        "bets {75,a}, raises {a}, max 2 raises (353,409 nodes)",
                         "turn": "turn precision study: 4-card board seed 2, top 50% each, pot 100 stack 300",
                         "river": "river HU: 5-card board seed 1, all 1081 combos each side, pot 100 stack 400",
                         "bench_spot": "reference bench_spot.json (Ks7h2d, 257 v 319)"}[args.workload],
            "board": cfg["board"], "arenas": ARENA_DESC[args.storage],
            "algo": "DCFR alpha 1.5 beta 0 gamma 2, alternating", "l2": "inputs larger than L2 (arenas GB-sized)",
            "parallelism": ("one spot sharded by turn card over the ranks, exact NCCL sums (strong scaling)"
                            if getattr(args, "shard", False) else "replica per GPU (weak scaling)"),
            "engine": getattr(args, "engine", "fused")}


def make_engine(g, host, args, world, rank, storage=None):
    """The engine of this rank: a replica of the whole spot, or with --shard
    this rank's shard of the one spot (NCCL sums between the ranks, captured
    in the iteration's graph; every rank builds it together)."""
    fmt = DEVICE_FORMAT[storage or args.storage]
    if not args.shard:
        return g.GpuSolver(host, device_format=fmt, engine=args.engine)
    nid = g.nccl_unique_id() if rank == 0 else None
    if world > 1:
        import torch.distributed as dist
        box = [nid]
        dist.broadcast_object_list(box, src=0)
        nid = box[0]
    return g.sharded_gpu_solver(host, rank, world, nid, device_format=fmt, engine=args.engine)


def run_ours(args, world, rank, local):
    import gtopen_b200 as g
    g.set_device(local)
    cfg = make_config(args.workload)
    t0 = time.perf_counter()
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage=HOST_STORAGE[args.storage], algo="dcfr", use_iso=True)
    build_s = time.perf_counter() - t0
    gpu = make_engine(g, host, args, world, rank)
    info = gpu.info()
    gpu.iterate(args.warmup)
    gpu.synchronize()
    barrier(world)
    clocks = Clocks(local)
    clocks.start()
    ms = gpu.time_iterations(args.steps)
    ck = clocks.stop()
    barrier(world)
    ms_max = allmax(ms, world)
    # replicas: every rank's iterations count; shards: the ranks run one spot
    value = (1 if args.shard else world) * args.steps / (ms_max / 1000.0)
    per_iter_s = ms / 1000.0 / args.steps
    peak, peak_kind = load_peak()
    achieved = info["iter_bytes"] / per_iter_s / 1e9
    prof = gpu.iterate_profiled()
    launches_per_iter = gpu.info()["iteration_kernels"]  # kernel nodes of the iteration's CUDA graph
    kinds = {g.KERNEL_NAMES[k]: round(prof.ms[k], 3) for k in range(7)}
    tot = sum(prof.ms) or 1.0
    dominant = max(range(7), key=lambda k: prof.ms[k])
    e_chk = gpu.exploitability(host)
    gpu.close()
    del gpu

    # end to end through the C ABI from host arenas
    e2e = None
    if not args.no_e2e:
        barrier(world)
        t = time.perf_counter()
        gpu2 = make_engine(g, host, args, world, rank)
        t_new = time.perf_counter()
        gpu2.iterate(args.steps)
        gpu2.synchronize()
        t_it = time.perf_counter()
        e = gpu2.exploitability(host)
        t_ex = time.perf_counter()
        gpu2.sync_to_cpu(host)
        gpu2.synchronize()
        t_end = time.perf_counter()
        dt = t_end - t
        split = {"new_s": t_new - t, "iterate_s": t_it - t_new, "exploitability_s": t_ex - t_it,
                 "sync_to_cpu_s": t_end - t_ex}
        dt_max = allmax(dt, world)
        b = HOST_BYTES[args.storage]
        arena_bytes = 2 * (spot.data_size[0] + spot.data_size[1]) * b
        up = gpu2.info()["upload_bytes"]
        e2e = {"value": (1 if args.shard else world) * args.steps / dt_max, "unit": "iter/s",
               "h2d_bytes_per_step": int(up / args.steps),
               "d2h_bytes_per_step": int((arena_bytes + 16) / args.steps),
               "includes": "GpuSolver::new (plan tables and, when the host solver has any, arenas uploaded; "
                           "a fresh solver's arenas are all zero and are not copied), %d iterations, "
                           "1 exploitability check (f64 read back), sync_to_cpu (every arena read back)" % args.steps,
               "split": {k: round(v, 3) for k, v in split.items()},
               "exploitability_pct_pot": e / cfg["tree"]["starting_pot"] * 100}
        gpu2.close()

    # time to the target on this workload (wall clock from GpuSolver::new,
    # exploitability checked on the GPU every check_every iterations), the
    # f32 arenas' run beside it, and the plain f32 kernels' iteration time
    ttt = ttt_f32 = plain = None
    if not args.no_ttt and args.shard:  # every rank takes part in a sharded solve
        ttt = time_to_target(g, cfg, args, factory=lambda host: make_engine(g, host, args, world, rank))
    elif not args.no_ttt and rank == 0:
        ttt = time_to_target(g, cfg, args)
        if args.storage != "f32":
            ttt_f32 = time_to_target(g, cfg, args, storage="f32")
        try:
            plain_ms = plain_f32_speed(g, cfg, 5)
        except g.GtobError as e:  # e.g. the plain engine's terminal slots exceed device memory
            plain_ms, plain = None, {"unavailable": str(e)}
        if plain_ms:
            plain = {"ms_per_iter": plain_ms, "iter_per_s": 1000.0 / plain_ms, "steps": 5,
                     "speedup_per_iter": (value / world) / (1000.0 / plain_ms)}
        if plain_ms and ttt_f32 and ttt_f32["reached"]:
            # the plain kernels would need the f32 run's iterations at their own speed
            plain["time_to_target_est_s"] = ttt_f32["iterations"] * plain_ms / 1000.0
            if ttt and ttt["reached"]:
                plain["speedup_time_to_target"] = plain["time_to_target_est_s"] / ttt["wall_s"]
    # time to 0.3% of the pot on the reference's own bench spot (bench_spot.json,
    # 1.25M nodes; exploitability checked every 10 iterations on the GPU, as
    # the reference CLI does), wall clock from GpuSolver::new
    ttt_spot = None
    if not args.no_spot_ttt and rank == 0 and not args.shard:
        ttt_spot = time_to_target(g, make_config("bench_spot"), args)
        ttt_spot["spot"] = "reference bench_spot.json (Ks7h2d, 257 v 319 hands, 1,245,971 nodes)"

    if rank != 0:
        return
    base = None
    if not args.no_cpu_baseline:
        r = cpu_baseline(cfg, args.storage, args.cpu_steps + 1, args.cpu_threads)
        timed = r["iter_s"][1:]  # the first iteration is the warm-up
        v = len(timed) / sum(timed)
        base = {"value": v, "unit": "iter/s", "cores": r["cores"], "kind": "port", "cpu_model": r["cpu_model"],
                "physical_cores": r["physical_cores"], "logical_cpus": r["logical_cpus"],
                "sample": "%d DCFR iterations of the same spot after 1 warm-up iteration on the CPU oracle "
                          "(reference cfr.rs semantics, %s arenas, pruning on, OpenMP over chance cards); "
                          "spot build %.1fs excluded" % (len(timed), ARENA_DESC[args.storage], r["build_s"])}
    line = {
        "metric": "CFR iterations/s (time-to-0.3%-pot exploitability & HBM GB/s vs peak)",
        "value": value, "unit": "iter/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "strong" if args.shard else "weak", "vs_baseline": None,
        "dtype": DTYPE[args.storage], "data": "synthetic (seeded spot)",
        "config": workload_config(args, cfg),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                     "traffic": MEASURED_TRAFFIC.get((args.workload, args.storage, args.engine)),
                     "kernel": "one CFR iteration (CUDA graph of all sweep kernels); dominant kind %s (%.0f%%)"
                               % (g.KERNEL_NAMES[dominant], 100.0 * prof.ms[dominant] / tot),
                     "algorithmic_bytes_per_iter": info["iter_bytes"]},
        "kernel_ms_profiled_iteration": kinds,
        "gpu_launches": launches_per_iter * args.steps,
        "clocks": ck,
        "e2e": e2e,
        "cpu_baseline": base,
        "tree": {"nodes": spot.num_nodes, "visited": info["visited_nodes"], "hands": spot.nh,
                 "levels": info["num_levels"], "device_gb": info["device_bytes"] / 1e9, "build_s": build_s},
        "exploitability_pct_pot_after": e_chk / cfg["tree"]["starting_pot"] * 100,
    }
    if ttt:
        line["time_to_target"] = ttt
    if ttt_f32:
        line["time_to_target_f32"] = ttt_f32
    if plain:
        line["plain_f32_kernels"] = plain
    if ttt_spot:
        line["time_to_target_bench_spot"] = ttt_spot
    print(json.dumps(line), flush=True)


def run_report(args, world, rank, local):
    """The flop report (184 suit-isomorphism classes of flops, the turn
    config's spot on each, 1-3 bet sizes per flop): every flop solved to the
    target through the batch API, `--report-workers` spots in flight on the
    GPU.  Flops are dealt round-robin over the ranks (strong scaling)."""
    import numpy as np

    import gtopen_b200 as g
    from concurrent.futures import ThreadPoolExecutor
    from gtopen_b200 import workloads as W
    g.set_device(local)
    pool = ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1)))
    build_s = 0.0

    def build_many(cs):  # the spot builds (tree, hands, river tables) are timed; drawing the ranges is not
        nonlocal build_s
        t = time.perf_counter()
        out = list(pool.map(g.Spot, cs))
        build_s += time.perf_counter() - t
        return out

    cfgs, spots = W.flop_report_spots(g.evaluate7, build_many, n=args.report_flops)
    mine = list(range(rank, len(spots), world))
    barrier(world)
    t1 = time.perf_counter()
    batch = g.Batch([spots[i] for i in mine], storage=HOST_STORAGE[args.storage],
                    device_format=DEVICE_FORMAT[args.storage], engine=args.engine, keep_solvers=False)
    persistent = args.batch_mode == "persistent"
    batch.run(max_iterations=args.ttt_max, target_pct=args.target, check_every=20, workers=args.report_workers,
              persistent=persistent, window=args.report_window)
    run_s = allmax(time.perf_counter() - t1, world)
    bstats = batch.stats() if persistent else None
    rows = batch.rows()
    bad = [r["error"] for r in rows if r["status"] != 0]
    if bad:
        raise RuntimeError("flop report: %d spot(s) failed: %s" % (len(bad), bad[0]))
    its = np.array([r["iterations"] for r in rows], np.float64)
    pct = np.array([r["exploit_pct"] for r in rows])
    reached = int((pct <= args.target).sum())
    stats = np.zeros(4)
    stats[:] = [its.sum(), reached, pct.max(), len(rows)]
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor(stats[:2].tolist() + [stats[3]], dtype=torch.float64)
        dist.all_reduce(t)
        m = torch.tensor([stats[2]], dtype=torch.float64)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        stats = np.array([t[0].item(), t[1].item(), m[0].item(), t[2].item()])
    n = len(spots)
    if rank != 0:
        return
    value = n / run_s * 3600.0
    sizes = [sp.num_nodes for sp in spots]
    line = {
        "metric": "flop report: flops/hour to %.1f%% pot exploitability" % args.target, "value": value,
        "unit": "flops/h", "n_gpus": world, "steps": n, "warmup": 0, "ms_per_step": 1000.0 * run_s / n,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": DTYPE[args.storage],
        "data": "synthetic (seeded spots)",
        "config": {"workload": "flop report: %d canonical flops (seed 4), turn-config ranges (top 50%% of 1176 "
                               "combos, weights U[0.2,1]), pot 100 stack 300, raise 2.5x, 2 raises, 1-3 bet sizes "
                               "from {33,50,75,125,a} (trees %d-%d nodes)" % (n, min(sizes), max(sizes)),
                   "arenas": ARENA_DESC[args.storage], "algo": "DCFR alpha 1.5 beta 0 gamma 2, alternating",
                   "check_every": 20, "max_iterations": args.ttt_max,
                   "batch": ("one persistent kernel launch per iteration of up to %d spots in flight "
                             "(a (spot, step, node tile) work queue)" % args.report_window if persistent else
                             "%d spots in flight, each on its own engine and CUDA graphs" % args.report_workers),
                   "parallelism": "flops dealt round-robin over ranks", "engine": args.engine},
        "report": {"reached_target": int(stats[1]), "flops": int(stats[3]), "iterations_total": int(stats[0]),
                   "worst_exploit_pct": float(stats[2]),
                   "median_iterations": float(np.median(its)), "median_spot_s": float(np.median(
                       [r["seconds"] for r in rows]))},
        "e2e": {"value": n / (run_s + build_s) * 3600.0, "unit": "flops/h",
                "includes": "spot builds (tree, hands, river tables; %.1f s on %d threads) + the batch run" % (
                    build_s, pool._max_workers),
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if bstats:
        line["persistent_kernel"] = bstats
        line["gpu_launches"] = int(bstats["launches"])
    if not args.no_cpu_baseline:
        mid = int(np.argsort(sizes)[len(sizes) // 2])
        r = cpu_baseline(cfgs[mid], args.storage, max(1, args.cpu_steps), args.cpu_threads)
        per_it = float(np.mean(r["iter_s"]))
        per_flop = r["build_s"] + per_it * float(np.median(its))
        line["cpu_baseline"] = {"value": 3600.0 / per_flop, "unit": "flops/h", "cores": r["cores"], "kind": "port",
                                "sample": "%d DCFR iteration(s) of the median-size flop (%d nodes) on the CPU "
                                          "oracle, times the GPU run's median iteration count (%d) plus its spot "
                                          "build: flops/hour extrapolated" % (len(r["iter_s"]), sizes[mid],
                                                                             int(np.median(its)))}
    print(json.dumps(line), flush=True)


def run_precision(args, world, rank, local):
    """The river (c1) and turn (c2) configurations: a fixed iteration count
    per arena format on the GPU, the GPU's own exploitability (f32 sweeps,
    f64 reduction) and the exploitability of the same average strategy under
    the oracle's f64 best response; iterations/s from CUDA events."""
    import numpy as np

    import gtopen_b200 as g
    from oracle import pyoracle as po
    g.set_device(local)
    if rank != 0:
        return
    out = {}
    for name, iters, fmts in (("river", 500, ("f32",)), ("turn", 1000, ("f32", "i16", "fp8"))):
        cfg = make_config(name)
        pot = cfg["tree"]["starting_pot"]
        ospot = po.Spot(cfg)
        for fmt in fmts:
            spot = g.Spot(cfg)
            host = g.Solver(spot, storage="f32", algo="dcfr", use_iso=True)
            gpu = g.GpuSolver(host, device_format=fmt, engine=args.engine)
            gpu.iterate(3)
            ms = gpu.time_iterations(iters - 3)
            e_gpu = gpu.exploitability(host) / pot * 100
            gpu.sync_to_cpu(host)
            host.ensure_symmetric()
            osv = po.Solver(ospot, compressed=False, algo="dcfr", use_iso=True, prune=False)
            for which in (0, 1):
                for p in (0, 1):
                    osv.set_arena(which, p, host.arena(which, p))
            e_f64 = osv.exploitability_f64() / pot * 100
            out["%s/%s" % (name, fmt)] = {
                "iterations": iters, "iter_per_s": (iters - 3) / (ms / 1000.0),
                "exploit_pct_gpu": e_gpu, "exploit_pct_f64_oracle": e_f64,
                "gpu_minus_f64_pct": e_gpu - e_f64, "nodes": spot.num_nodes, "hands": list(spot.nh)}
            gpu.close()
    line = {"metric": "configs c1 (river) and c2 (turn): exploitability after a fixed iteration count per arena "
                      "format, GPU vs f64 best-response oracle", "value": out["turn/i16"]["iter_per_s"],
            "unit": "iter/s", "n_gpus": 1, "steps": 1000, "warmup": 3, "higher_is_better": True,
            "data": "synthetic (seeded spots)", "configs": out}
    print(json.dumps(line), flush=True)


BF16_FALLBACK = 1590.0  # TFLOP/s, burst


def load_bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return BF16_FALLBACK, "fallback"


def run_leaf(args, world, rank, local):
    """The depth-limited configuration: turn spots of the flop solved by the
    plain engine (the training set), the leaf network trained on the device,
    depth-limited solves with the trained and an untrained network, and each
    resulting flop strategy checked on the full tree (player p's flop locked,
    the rest re-solved: p's loss of game value, % pot).  Also the tcgen05
    product's throughput against the bf16 peak."""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor

    import gtopen_b200 as g
    from gtopen_b200 import leafdata as LD
    g.set_device(local)
    if rank != 0:
        return
    t_all = time.perf_counter()
    cfg = LD.dl_flop_spot(g.evaluate7)
    spot = g.Spot(cfg)
    _, pots, stacks, _ = g.dl_plan(spot)  # the leaves of the host-built plan
    leaf_pots = sorted(set((float(a), float(b)) for a, b in zip(pots, stacks)))
    pool = ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1)))
    t = time.perf_counter()
    X, T, M, info = LD.training_set(g, cfg, leaf_pots, args.leaf_spots, seed=1, workers=16, build_pool=pool)
    gen_s = time.perf_counter() - t
    nval = max(128, args.leaf_spots // 10)
    Xt, Tt, Mt = X[nval:], T[nval:], M[nval:]
    Xv, Tv, Mv = X[:nval], T[:nval], M[:nval]
    net = g.LeafNet(LD.LEAF_IN, 1024, 3, LD.LEAF_OUT, seed=7)
    untrained = g.LeafNet(LD.LEAF_IN, 1024, 3, LD.LEAF_OUT, seed=7)
    val0 = net.gradients(Xv, Tv, Mv)
    t = time.perf_counter()
    losses = net.train(Xt, Tt, Mt, epochs=args.leaf_epochs, batch=256, lr=args.leaf_lr, seed=3)
    train_s = time.perf_counter() - t
    val1 = net.gradients(Xv, Tv, Mv)
    rows_seen = args.leaf_epochs * (len(Xt) // 256) * 256
    dims = [(2816, 1024), (1024, 1024), (1024, 1024), (1024, 2688)]
    fwd = sum(2.0 * i * o for i, o in dims)
    flops = rows_seen * (3.0 * fwd - 2.0 * 2816 * 1024)  # forward, dW, dX (no dX into the inputs)
    # the product alone, operands resident: the forward pass's widest shape at the training batch
    peak, peak_kind = load_bf16_peak()
    gm, gn, gk = 4096, 1024, 2816
    gms = g.gemm_time_ms(gm, gn, gk, reps=50)
    g_tflops = 2.0 * gm * gn * gk / (gms / 1000.0) / 1e12
    check = LD.FullTreeCheck(g, cfg, iterations=args.leaf_check_iters)
    res = {}
    for name, n in (("trained", net), ("untrained", untrained)):
        r = LD.depth_limited_or_full(g, cfg, n, check, dl_iterations=args.leaf_dl_iters)
        r.pop("strategies")
        res[name] = r
    # the non-learned leaf: the flop solved with the turn and river checked
    # down (showdown equity of the ranges reaching each turn), judged the same way
    t = time.perf_counter()
    cd = LD.checkdown_flop_strategies(g, cfg, iterations=args.leaf_dl_iters)
    c0, c1, cex = check.loss(cd)
    res["checkdown"] = {"loss_pct": [c0, c1], "loss_sum_pct": c0 + c1, "locked_solve_exploit_pct": cex,
                        "solve_s": time.perf_counter() - t}
    line = {"metric": "depth-limited flop solve (config 5): flop-strategy loss vs the full-tree solve, "
                      "trained vs untrained turn-leaf network",
            "value": res["trained"]["loss_sum_pct"], "unit": "% pot (sum over players)", "n_gpus": 1,
            "higher_is_better": False, "dtype": "bf16 (network), f32 (solve)", "data": "synthetic (seeded spots)",
            "config": {"workload": "dl_flop c5: flop %s, 1.94M-node full tree cut at 11 turn leaves, "
                                   "network 2705-1024x3-2652" % cfg["board"],
                       "training_spots": len(Xt), "validation_spots": nval},
            "trained": res["trained"], "untrained": res["untrained"], "checkdown_leaf": res["checkdown"],
            "answer_path": res["trained"]["path"], "fallback_threshold_pct": LD.FALLBACK_PCT,
            "full_solve": {"iterations": check.iterations, "exploit_pct": check.full_exploit},
            "training": {"spots_generated": args.leaf_spots, "generate_s": gen_s,
                         "turn_solve_exploit_pct_mean": float(info["exploit_pct"].mean()),
                         "epochs": args.leaf_epochs, "train_s": train_s, "loss_first": float(losses[0]),
                         "loss_last": float(losses[-1]), "val_loss_before": val0, "val_loss_after": val1,
                         "tflops": flops / train_s / 1e12},
            "roofline": {"bound": "tensor", "kernel": "k_gemm_tn %dx%dx%d" % (gm, gn, gk), "achieved": g_tflops,
                         "peak": peak, "unit": "TFLOP/s", "frac": g_tflops / peak,
                         "peak_kind": peak_kind + " bf16 dense", "ms": gms},
            "wall_s": time.perf_counter() - t_all}
    print(json.dumps(line), flush=True)


def time_to_target(g, cfg, args, storage=None, engine=None, factory=None):
    storage = storage or args.storage
    engine = engine or args.engine
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage=HOST_STORAGE[storage], algo="dcfr", use_iso=True)
    t = time.perf_counter()
    if factory is not None:
        gpu = factory(host)
    else:
        gpu = g.GpuSolver(host, device_format=DEVICE_FORMAT[storage], engine=engine)
    pot = cfg["tree"]["starting_pot"]
    pct = None
    while gpu.iteration < args.ttt_max:
        gpu.iterate(args.check_every)
        pct = gpu.exploitability(host) / pot * 100
        if pct <= args.target:
            break
    gpu.synchronize()
    dt = time.perf_counter() - t
    it = gpu.iteration
    gpu.close()
    return {"target_pct_pot": args.target, "reached": pct is not None and pct <= args.target, "iterations": it,
            "wall_s": dt, "final_pct_pot": pct, "check_every": args.check_every, "arenas": ARENA_DESC[storage],
            "engine": engine}


def plain_f32_speed(g, cfg, steps):
    """The plain f32 kernels (one launch per node kind and level, f32 arenas)
    on the same spot: device time per iteration."""
    spot = g.Spot(cfg)
    host = g.Solver(spot, storage="f32", algo="dcfr", use_iso=True)
    gpu = g.GpuSolver(host, engine="plain")
    gpu.iterate(2)
    gpu.synchronize()
    ms = gpu.time_iterations(steps) / steps
    gpu.close()
    return ms


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="flop",
                    choices=["flop", "flop_narrow", "turn", "river", "bench_spot", "report", "precision", "leaf"])
    ap.add_argument("--leaf-spots", type=int, default=2048, help="turn spots solved for the leaf network")
    ap.add_argument("--leaf-epochs", type=int, default=60)
    ap.add_argument("--leaf-lr", type=float, default=3e-4)
    ap.add_argument("--leaf-dl-iters", type=int, default=400)
    ap.add_argument("--leaf-check-iters", type=int, default=400)
    ap.add_argument("--report-flops", type=int, default=184)
    ap.add_argument("--report-workers", type=int, default=8)
    ap.add_argument("--batch-mode", default="concurrent", choices=["persistent", "concurrent"],
                    help="report: an engine per spot in flight (the faster here), or one persistent kernel over them")
    ap.add_argument("--report-window", type=int, default=16, help="report: spots in flight on the persistent kernel")
    ap.add_argument("--storage", default="i16sr", choices=["i16sr", "compressed", "f32", "fp8"])
    ap.add_argument("--engine", default="staged", choices=["fused", "plain", "warp", "fused32", "staged", "staged_river"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="split the one spot over the ranks by turn card (NCCL sums) instead of a replica per rank")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=3, help="timed CPU-oracle iterations (after one warm-up)")
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--no-ttt", action="store_true",
                    help="skip the time-to-target runs on the workload (i16 and f32 arenas) and the plain f32 timing")
    ap.add_argument("--target", type=float, default=0.3)
    ap.add_argument("--check-every", type=int, default=10)
    ap.add_argument("--ttt-max", type=int, default=2000)
    ap.add_argument("--no-spot-ttt", action="store_true", help="skip the time-to-target run on the bench spot")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference" and args.workload in ("report", "precision", "leaf"):
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the %s workload has no reference-arm run "
                                  "(the flop report extrapolates its CPU baseline from sampled oracle iterations; "
                                  "the precision runs compare with the oracle's f64 best response)" % args.workload}),
                      flush=True)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "report":
            run_report(args, world, rank, local)
        elif args.workload == "precision":
            run_precision(args, world, rank, local)
        elif args.workload == "leaf":
            run_leaf(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
