#include "batch.hpp"

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cmath>
#include <thread>

#include "../kernels/engine.hpp"

namespace gtob {

std::vector<double> valid_opp_sum(const Spot& spot, int p, const float* reach_o) {
    const Hands& ho = spot.hands[1 - p];
    double t = 0.0, s[52] = {0.0};
    for (size_t j = 0; j < ho.size(); j++) {
        const double r = (double)reach_o[j];
        t += r;
        s[ho.c1[j]] += r;
        s[ho.c2[j]] += r;
    }
    const Hands& hp = spot.hands[p];
    std::vector<double> out(hp.size());
    for (size_t i = 0; i < hp.size(); i++) {
        const uint32_t same = spot.same[p][i];
        const double same_r = same != kSentinel ? (double)reach_o[same] : 0.0;
        out[i] = t - s[hp.c1[i]] - s[hp.c2[i]] + same_r;
    }
    return out;
}

static void solve_one(HostSolver& host, bool sync, int device_format, int engine, uint32_t max_iterations,
                      double target_pct, uint32_t check_every, BatchRow& row) {
    const auto t0 = std::chrono::steady_clock::now();
    const Spot& sp = *host.spot;
    const double pot = sp.config.tree.starting_pot;
    GpuEngine eng(host, device_format, engine);
    double pct = NAN;
    for (;;) {
        eng.iterate(1);
        const uint32_t it = eng.iteration();
        if (it % check_every == 0 || it >= max_iterations) {
            pct = eng.exploitability(host) / pot * 100.0;
            if (pct <= target_pct || it >= max_iterations) break;
        }
    }
    // root EVs of the average strategies (solve_cli.rs:176-188 over node_view
    // at the root, query.rs:490-600): ev(h) = cfv(h) / valid(h) + put, averaged
    // over the hands with valid > 1e-9, weighted by their reach (the range)
    for (int p = 0; p < 2; p++) {
        const Hands& h = sp.hands[p];
        std::vector<float> cfv(h.size());
        eng.root_cfv(p, 1, cfv.data());
        const std::vector<double> valid = valid_opp_sum(sp, p, sp.hands[1 - p].w.data());
        const double put = p == 0 ? sp.tree.put0[0] : sp.tree.put1[0];
        double n = 0.0, d = 0.0;
        for (size_t i = 0; i < h.size(); i++) {
            if (!(valid[i] > 1e-9)) continue;
            const float ev = (float)((double)cfv[i] / valid[i] + put);
            n += (double)ev * (double)h.w[i];
            d += (double)h.w[i];
        }
        row.ev[p] = n / d;
        row.root_cfv[p] = std::move(cfv);
    }
    if (sync) eng.sync_to_cpu(host, false);
    row.iterations = eng.iteration();
    row.exploit_pct = pct;
    row.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void run_batch(const std::vector<std::shared_ptr<Spot>>& spots, const std::vector<HostSolver*>& solvers, int storage,
               int algo, bool use_iso, int device_format, int engine, uint32_t max_iterations, double target_pct,
               uint32_t check_every, int workers, std::vector<BatchRow>& rows) {
    if (check_every == 0) throw Error("invalid argument: check_every must be positive");
    if (solvers.size() != spots.size()) throw Error("invalid argument: one solver slot per spot");
    rows.assign(solvers.size(), BatchRow{});
    int device = 0;
    const cudaError_t rc = cudaGetDevice(&device);
    if (rc != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(rc));
    std::atomic<size_t> next{0};
    auto work = [&] {
        const cudaError_t r = cudaSetDevice(device);
        for (size_t i; (i = next.fetch_add(1)) < solvers.size();) {
            try {
                if (r != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(r));
                if (solvers[i]) {
                    solve_one(*solvers[i], true, device_format, engine, max_iterations, target_pct, check_every, rows[i]);
                } else {
                    HostSolver shell(spots[i], storage, algo, use_iso, false);
                    solve_one(shell, false, device_format, engine, max_iterations, target_pct, check_every, rows[i]);
                }
            } catch (const std::exception& e) {
                rows[i].error = e.what();
                rows[i].error = rows[i].error.empty() ? "unknown error" : rows[i].error;
            }
        }
    };
    const int nw = std::max(1, std::min<int>(workers, (int)solvers.size()));
    std::vector<std::thread> ts;
    for (int w = 1; w < nw; w++) ts.emplace_back(work);
    work();
    for (auto& t : ts) t.join();
}

}  // namespace gtob
