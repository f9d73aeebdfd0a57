#include "batch.hpp"

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
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

// The end of one spot's solve: root EVs of the average strategies
// (solve_cli.rs:176-188 over node_view at the root, query.rs:490-600):
// ev(h) = cfv(h) / valid(h) + put, averaged over the hands with valid >
// 1e-9, weighted by their reach (the range); then the host solver synced.
static void finish_one(GpuEngine& eng, HostSolver& host, bool sync, double pct,
                       std::chrono::steady_clock::time_point t0, BatchRow& row) {
    const Spot& sp = *host.spot;
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

static void solve_one(HostSolver& host, bool sync, int device_format, int engine, uint32_t max_iterations,
                      double target_pct, uint32_t check_every, BatchRow& row) {
    const auto t0 = std::chrono::steady_clock::now();
    const double pot = host.spot->config.tree.starting_pot;
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
    finish_one(eng, host, sync, pct, t0, row);
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

// ---------------------------------------------------------------------------
// The batch on the persistent kernel (BatchKernel): a window of spots whose
// iterations all run in one launch per iteration.

namespace {

// Batch shapes picked per (arena format, size class) from timed iterations
// and kept in a small text file ("fmt class tile ctas" per line): the path
// in GTOB_TUNE_CACHE, else $HOME/.cache/gtob/batch_shapes.txt; without a
// writable path the choices live in this process only.
class ShapeCache {
  public:
    static ShapeCache& get() {
        static ShapeCache c;
        return c;
    }
    bool find(int fmt, int cls, BatchShape* out) {
        std::lock_guard<std::mutex> lk(mu_);
        load();
        auto it = m_.find({fmt, cls});
        if (it == m_.end()) return false;
        *out = it->second;
        return true;
    }
    void put(int fmt, int cls, const BatchShape& s) {
        std::lock_guard<std::mutex> lk(mu_);
        load();
        m_[{fmt, cls}] = s;
        const std::string p = path();
        if (p.empty()) return;
        for (size_t pos = 1; (pos = p.find('/', pos)) != std::string::npos; pos++) mkdir_one(p.substr(0, pos));
        const std::string tmp = p + ".tmp";
        {
            std::ofstream f(tmp);
            if (!f) return;
            for (auto& kv : m_)
                f << kv.first.first << ' ' << kv.first.second << ' ' << kv.second.tile << ' ' << kv.second.ctas_per_sm
                  << '\n';
            if (!f) return;
        }
        std::rename(tmp.c_str(), p.c_str());
    }
    static std::string path() {
        const char* e = std::getenv("GTOB_TUNE_CACHE");
        if (e) return e;
        const char* h = std::getenv("HOME");
        return h ? std::string(h) + "/.cache/gtob/batch_shapes.txt" : std::string();
    }

  private:
    static void mkdir_one(const std::string& d);
    void load() {  // (again when the path changed)
        const std::string p = path();
        if (loaded_ && p == loaded_path_) return;
        loaded_ = true;
        loaded_path_ = p;
        m_.clear();
        if (p.empty()) return;
        std::ifstream f(p);
        int fmt, cls, tile, ctas;
        while (f >> fmt >> cls >> tile >> ctas)
            if (tile >= 1 && tile <= 64 && ctas >= 0 && ctas <= 64) m_[{fmt, cls}] = BatchShape{tile, ctas};
    }
    std::mutex mu_;
    bool loaded_ = false;
    std::string loaded_path_;
    std::map<std::pair<int, int>, BatchShape> m_;
};

}  // namespace
}  // namespace gtob

#include <sys/stat.h>

namespace gtob {
namespace {
void ShapeCache::mkdir_one(const std::string& d) { ::mkdir(d.c_str(), 0755); }

// The size class of a set of spots: log2 of its total tree nodes.
int size_class(const std::vector<std::shared_ptr<Spot>>& spots, const std::vector<size_t>& idx) {
    double n = 0.0;
    for (size_t i : idx) n += (double)spots[i]->tree.size();
    return n > 1.0 ? (int)std::floor(std::log2(n)) : 0;
}

bool trace_on() {
    static const bool on = std::getenv("GTOB_BATCH_TRACE") != nullptr;
    return on;
}
#define BTRACE(...)                                  \
    do {                                             \
        if (trace_on()) {                            \
            std::fprintf(stderr, "[batch] " __VA_ARGS__); \
            std::fflush(stderr);                     \
        }                                            \
    } while (0)

struct Live {
    size_t idx;
    std::unique_ptr<HostSolver> shell;  // when the batch keeps no solver for this spot
    HostSolver* host;
    std::unique_ptr<GpuEngine> eng;
    std::chrono::steady_clock::time_point t0;
};
}  // namespace

void run_batch_persistent(const std::vector<std::shared_ptr<Spot>>& spots, const std::vector<HostSolver*>& solvers,
                          int storage, int algo, bool use_iso, int device_format, uint32_t max_iterations,
                          double target_pct, uint32_t check_every, int window, std::vector<BatchRow>& rows,
                          BatchRunStats* stats) {
    if (check_every == 0) throw Error("invalid argument: check_every must be positive");
    if (solvers.size() != spots.size()) throw Error("invalid argument: one solver slot per spot");
    if (window < 1) throw Error("invalid argument: the window holds at least one spot");
    rows.assign(solvers.size(), BatchRow{});
    BatchRunStats st;
    int device = 0;
    {
        // the device's context bound to this thread before any other thread
        // builds engines: the engines' streams and buffers must belong to the
        // context this thread launches in, for the whole run
        cudaError_t rc = cudaGetDevice(&device);
        if (rc == cudaSuccess) rc = cudaSetDevice(device);
        if (rc != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(rc));
    }
    // builder thread: engines for the spots in order, at most kPrefetch built
    // ahead of the window, and each only once the device has room for it --
    // its size predicted from the bytes per tree node of the engines built so
    // far -- unless nothing else holds device memory (a spot whose engine
    // fails gets its error row)
    constexpr size_t kPrefetch = 2;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Live> ready;
    size_t built = 0;   // spots the builder has finished with (engine ready or error row)
    size_t held = 0;    // engines alive (ready or in the window)
    bool stop = false;
    double bytes_per_node = 0.0;  // of the engines built so far (0: none yet)
    std::thread builder([&] {
        const cudaError_t r = cudaSetDevice(device);
        for (size_t i = 0; i < solvers.size(); i++) {
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    if (stop) return;
                    if (ready.size() < kPrefetch) {
                        size_t fr = 0, tot = 0;
                        const double need = bytes_per_node * (double)spots[i]->tree.size() * 1.15 + (1ull << 30);
                        if (held == 0 || bytes_per_node <= 0.0 || (cudaMemGetInfo(&fr, &tot) == cudaSuccess && (double)fr >= need))
                            break;
                    }
                    cv.wait_for(lk, std::chrono::milliseconds(20));
                }
            }
            Live L;
            L.idx = i;
            L.t0 = std::chrono::steady_clock::now();
            try {
                if (r != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(r));
                if (solvers[i]) {
                    L.host = solvers[i];
                } else {
                    L.shell = std::make_unique<HostSolver>(spots[i], storage, algo, use_iso, false);
                    L.host = L.shell.get();
                }
                L.eng = std::make_unique<GpuEngine>(*L.host, device_format, kEngineStaged);
                const std::string why = BatchKernel::unsupported(*L.eng);
                if (!why.empty()) throw Error("invalid argument: " + why);
            } catch (const std::exception& e) {
                rows[i].error = e.what();
                if (rows[i].error.empty()) rows[i].error = "unknown error";
                L.eng.reset();
            }
            BTRACE("built spot %zu engine %p err '%s'\n", i, (void*)L.eng.get(), rows[i].error.c_str());
            std::lock_guard<std::mutex> lk(mu);
            if (L.eng) {
                const double bpn = (double)L.eng->device_bytes() / (double)std::max<size_t>(spots[i]->tree.size(), 1);
                bytes_per_node = std::max(bytes_per_node, bpn);
                held++;
                ready.push_back(std::move(L));
            }
            built++;
            cv.notify_all();
        }
        // stays until the run ends (the thread that built the engines outlives them)
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop; });
    });
    struct Join {
        std::thread& t;
        std::mutex& m;
        std::condition_variable& c;
        bool& s;
        ~Join() {
            {
                std::lock_guard<std::mutex> lk(m);
                s = true;
            }
            c.notify_all();
            if (t.joinable()) t.join();
        }
    } join{builder, mu, cv, stop};

    BatchKernel bk;
    std::vector<Live> live;
    bool changed = true;
    // autotuning state: candidates timed one real iteration each (the
    // shape does not change any result, so trial iterations are ordinary ones)
    std::vector<BatchShape> cand;
    std::vector<double> cand_ms;
    size_t cand_next = 0;
    int cls = -1, fmt = -1;
    const char* phase = "start";
    try {
    for (;;) {
        {  // admit built spots while the window has room
            std::unique_lock<std::mutex> lk(mu);
            // an empty window (the start) fills up first, so that the first
            // set -- the one whose size class gets tuned -- is a full one
            // (or as full as device memory allows)
            if (live.empty()) {
                while (live.size() < (size_t)window && built < solvers.size()) {
                    if (ready.empty()) {
                        cv.wait_for(lk, std::chrono::milliseconds(20));
                        // the builder waits for room that only this window's
                        // start can give: start with what is there
                        size_t fr = 0, tot = 0;
                        if (ready.empty() && !live.empty() && cudaMemGetInfo(&fr, &tot) == cudaSuccess &&
                            (double)fr < bytes_per_node * (double)spots[built]->tree.size() * 1.15 + (1ull << 30))
                            break;
                        continue;
                    }
                    live.push_back(std::move(ready.front()));
                    ready.pop_front();
                    changed = true;
                    cv.notify_all();
                }
            }
            while (live.size() < (size_t)window && !ready.empty()) {
                live.push_back(std::move(ready.front()));
                ready.pop_front();
                changed = true;
            }
            cv.notify_all();
            if (live.empty() && ready.empty() && built == solvers.size()) break;
        }
        if (live.empty()) continue;
        if (changed) {
            std::vector<GpuEngine*> ptr;
            std::vector<size_t> idx;
            for (auto& L : live) {
                ptr.push_back(L.eng.get());
                idx.push_back(L.idx);
            }
            const int c = size_class(spots, idx);
            const int f = live[0].eng->format();
            BatchShape shape = bk.shape();
            if (c != cls || f != fmt) {  // a new size class: its cached shape, or tune it
                cls = c;
                fmt = f;
                cand.clear();
                cand_ms.clear();
                cand_next = 0;
                if (!ShapeCache::get().find(fmt, cls, &shape)) {
                    const int occ = 0;  // 0: as many CTAs per SM as fit
                    for (int tile : {1, 2, 4, 8})
                        for (int ctas : {occ, 1}) cand.push_back(BatchShape{tile, ctas});
                }
            }
            if (cand_next < cand.size()) shape = cand[cand_next];
            phase = "configure";
            for (auto& L : live) BTRACE("set: spot %zu engine %p it %u\n", L.idx, (void*)L.eng.get(), L.eng->iteration());
            bk.configure(ptr, shape);
            changed = false;
        }
        // one iteration of every live spot (a trial of the next candidate
        // shape while the class is being tuned: the shape changes no result,
        // so a trial iteration is an ordinary one)
        if (cand_next < cand.size()) {
            phase = "configure a trial shape";
            bk.configure_shape(cand[cand_next]);
            phase = "trial iteration";
            const double ms = bk.time_iterations(1);
            st.kernel_ms += ms;
            // per node record: the set may shrink while the class is tuned
            cand_ms.push_back(ms / (double)std::max<uint64_t>(bk.records(), 1));
            if (++cand_next == cand.size()) {
                size_t best = 0;
                for (size_t k = 1; k < cand.size(); k++)
                    if (cand_ms[k] < cand_ms[best]) best = k;
                bk.configure_shape(cand[best]);
                ShapeCache::get().put(fmt, cls, cand[best]);
                st.tuned++;
            }
        } else {
            phase = "iteration";
            st.kernel_ms += bk.time_iterations(1);
        }
        st.launches++;
        // checks (solve_quiet's rule), in parallel: each engine's evaluation
        // sweeps run on its own stream
        std::vector<size_t> chk;
        for (size_t k = 0; k < live.size(); k++) {
            const uint32_t it = live[k].eng->iteration();
            if (it % check_every == 0 || it >= max_iterations) chk.push_back(k);
        }
        if (chk.empty()) continue;
        std::vector<double> pct(chk.size(), NAN);
        std::vector<std::string> err(chk.size());
        parallel_for(chk.size(), [&](size_t j) {
            int stage = 0;
            try {
                const cudaError_t r = cudaSetDevice(device);
                if (r != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(r));
                Live& L = live[chk[j]];
                BTRACE("check spot %zu engine %p it %u\n", L.idx, (void*)L.eng.get(), L.eng->iteration());
                pct[j] = L.eng->exploitability(*L.host) / spots[L.idx]->config.tree.starting_pot * 100.0;
                stage = 1;
                if (pct[j] <= target_pct || L.eng->iteration() >= max_iterations)
                    finish_one(*L.eng, *L.host, L.shell == nullptr, pct[j], L.t0, rows[L.idx]);
            } catch (const std::exception& e) {
                err[j] = std::string(e.what()) + (stage ? " (root values and sync)" : " (exploitability check)");
                if (err[j].empty()) err[j] = "unknown error";
            }
        });
        std::vector<bool> drop(live.size(), false);
        for (size_t j = 0; j < chk.size(); j++) {
            Live& L = live[chk[j]];
            if (!err[j].empty()) {
                rows[L.idx].error = err[j];
                drop[chk[j]] = true;
            } else if (pct[j] <= target_pct || L.eng->iteration() >= max_iterations) {
                drop[chk[j]] = true;
            }
        }
        if (std::find(drop.begin(), drop.end(), true) != drop.end()) {
            std::vector<Live> keep;
            for (size_t k = 0; k < live.size(); k++) {
                if (drop[k]) {
                    BTRACE("drop spot %zu engine %p\n", live[k].idx, (void*)live[k].eng.get());
                    continue;
                }
                keep.push_back(std::move(live[k]));
            }
            phase = "release finished spots";
            bk.configure({}, bk.shape());  // the kernel's set holds no engine about to be freed
            const size_t freed = live.size() - keep.size();
            live = std::move(keep);        // the finished engines are freed here
            changed = true;
            {
                std::lock_guard<std::mutex> lk(mu);
                held -= freed;
            }
            cv.notify_all();
        }
    }
    } catch (const std::exception& e) {
        throw Error(std::string(e.what()) + " [persistent batch: " + phase + "]");
    }
    const BatchShape s = bk.shape();
    st.tile = s.tile;
    st.ctas_per_sm = s.ctas_per_sm;
    st.grid = bk.grid();
    if (stats) *stats = st;
}

}  // namespace gtob
