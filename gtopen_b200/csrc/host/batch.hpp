// Many spots on one GPU at once: the reference's batch report
// (solve_cli.rs:125-215, run per board with solve_quiet, solve_cli.rs:338-362)
// with the spots solved side by side instead of one after another.  Worker
// threads each take the next spot, build its GPU engine (own streams, own
// CUDA graphs), solve it to the target, read its root EVs and sync it back;
// the engines of different workers run concurrently on the device, which a
// single spot of a few thousand nodes cannot fill.
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "solver.hpp"

namespace gtob {

struct BatchRow {
    std::string error;  // empty: solved
    uint32_t iterations = 0;
    double exploit_pct = 0.0;  // exploitability, % of the starting pot
    double seconds = 0.0;      // wall time of this spot: engine build, solve, EVs, sync
    double ev[2] = {0.0, 0.0};  // reach-weighted root EV per player, pot-share (solve_cli.rs:176-188)
    std::vector<float> root_cfv[2];  // per hand, the root's counterfactual values of the average strategies
};

// Runs solve_quiet's loop (one iteration at a time, exploitability when the
// iteration is a multiple of check_every or reaches max_iterations, stop at
// target_pct or max_iterations) for every spot, with up to `workers` spots in
// flight; rows[i] describes spots[i].  A spot with a host solver in
// solvers[i] is synced back into it; one without (nullptr) is solved against a
// host solver that holds no arenas, built and dropped by its worker, so the
// batch's host memory stays bounded by the spots in flight.  Errors stay in
// their row.  Must be called with the target device current.
void run_batch(const std::vector<std::shared_ptr<Spot>>& spots, const std::vector<HostSolver*>& solvers, int storage,
               int algo, bool use_iso, int device_format, int engine, uint32_t max_iterations, double target_pct,
               uint32_t check_every, int workers, std::vector<BatchRow>& rows);

// The batch on ONE persistent kernel (BatchKernel, cfr_batch.cuh): up to
// `window` spots in flight, every iteration of all of them one launch; spots
// leave at their checks (the same rule and the same per-spot iterations as
// run_batch, so each row equals the spot solved alone) and a builder thread
// keeps the next engines ready.  Shapes (records per ticket, CTAs per SM)
// are tuned per size class from timed iterations and cached on disk
// (GTOB_TUNE_CACHE or ~/.cache/gtob/batch_shapes.txt).  Staged engines only.
struct BatchRunStats {
    uint64_t launches = 0;   // batched iterations (one kernel launch each)
    double kernel_ms = 0.0;  // device time of those launches (CUDA events)
    int tuned = 0;           // size classes tuned in this run
    int tile = 0, ctas_per_sm = 0, grid = 0;  // the last shape used
};
void run_batch_persistent(const std::vector<std::shared_ptr<Spot>>& spots, const std::vector<HostSolver*>& solvers,
                          int storage, int algo, bool use_iso, int device_format, uint32_t max_iterations,
                          double target_pct, uint32_t check_every, int window, std::vector<BatchRow>& rows,
                          BatchRunStats* stats);

// Per-hand compatible opponent reach mass (query.rs:463-488), f64.
std::vector<double> valid_opp_sum(const Spot& spot, int p, const float* reach_o);

}  // namespace gtob
