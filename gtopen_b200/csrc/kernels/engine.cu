// Level-synchronous discounted-CFR engine for sm_100a: host side.
//
// One iteration = for traverser p in {0, 1}: a down sweep writing reach
// vectors level by level, then an up sweep folding counterfactual values back
// to the root with the DCFR / CFR+ / PCFR+ regret and strategy-sum update --
// the work split of the reference's gpu/kernels.cu and gpu/mod.rs:622-841,
// re-designed for B200 (device code in cfr_kernels.cuh):
//   * work items carry precomputed slots (plan.hpp); reach and cfv vectors
//     live in compact slots;
//   * FUSED engine (default): fold and showdown children are evaluated in
//     shared memory by their parent's up-sweep kernel (all-in runouts by the
//     river chance node's kernel), so terminals -- two thirds of all nodes --
//     never write or read a vector in HBM and need no launches of their own;
//     the PLAIN engine keeps one kernel launch per terminal level;
//   * arenas are hand-major per node, f32 or 16-bit with a per-node scale
//     (requantised in-kernel after a block max), matching cfr.rs:297-409;
//   * discounts are computed on the device in f64 from a device iteration
//     counter, so one captured CUDA graph replays every iteration.
// Summation orders equal the reference CPU engine's, and the CUDA code is
// compiled with -fmad=false (every multiply and add rounds separately, as the
// reference's f32 arithmetic does).
#include <cuda_runtime.h>

#include "leafnet.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <istream>
#include <map>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <unordered_map>
#include <string>
#include <vector>

#include "cfr_kernels.cuh"
#include "cfr_staged.cuh"
#include "cfr_river.cuh"
#include "cfr_batch.cuh"
#include "engine.hpp"

namespace gtob {

const char* const kKernelNames[7] = {"copy_root", "down_action", "down_chance", "up_fold",
                                     "up_show",   "up_chance",   "up_action"};

#define CK(x)                                                                                           \
    do {                                                                                                \
        cudaError_t e_ = (x);                                                                           \
        if (e_ != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(e_) + " at " #x); \
    } while (0)

static thread_local uint64_t g_uploaded = 0;  // host-to-device bytes of the engine being built
template <class V>
static typename V::value_type* dupload(const V& v, std::vector<void*>& owned, size_t* bytes) {
    using T = typename V::value_type;
    T* p = nullptr;
    const size_t n = std::max<size_t>(v.size(), 1);
    CK(cudaMalloc(&p, n * sizeof(T)));
    owned.push_back(p);
    *bytes += n * sizeof(T);
    if (!v.empty()) CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    g_uploaded += v.size() * sizeof(T);
    return p;
}
static void* dalloc(size_t bytes, std::vector<void*>& owned, size_t* total) {
    void* p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
    owned.push_back(p);
    *total += bytes;
    CK(cudaMemset(p, 0, std::max<size_t>(bytes, 16)));
    return p;
}
// A kernel's dynamic shared-memory limit is per function and process: raise it
// to what this engine launches with, never lower it (engines of different
// spots run side by side in a batch).  The default limit is 48 KB minus the
// kernel's static shared memory, so the attribute is set for any size.
static void set_smem(const void* fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> set;  // (device, kernel) -> limit set
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = set[{dev, fn}];
    if (bytes <= cur) return;
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
}

struct EngineImpl {
    const Spot* spot;
    Plan plan;
    int fmt = kFmtF32;
    int algo = kDcfr;
    bool pcfr = false;
    bool wide = false;  // some node has more than 8 actions: use the 32-wide kernels
    bool term64 = false;  // terminal sums in f64 (plain engine, or fused on request)
    bool warp = false;    // warp-per-node action kernels, fold children in place
    bool staged = false;  // staged (bulk-copy) node kernels, fold children in place
    bool reach_valid = false;  // reach slots hold the current strategies' reach (see prime)
    uint32_t iteration = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;  // terminals of a captured sweep
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::vector<cudaEvent_t> ev_term;  // per level: that level's terminals are done
    std::vector<void*> owned;
    size_t bytes = 0;
    uint64_t uploaded = 0;  // host-to-device bytes copied by the constructor
    Dev d{};
    Arenas ar{};
    ActItem* act = nullptr;
    EdgeItem* edge = nullptr;
    FoldItem* fold = nullptr;
    ShowItem* show = nullptr;
    ShowBatch* show_batch = nullptr;
    ChanceItem* chance = nullptr;
    XNode* xnodes[2] = {nullptr, nullptr};
    std::vector<XNode> hx[2];
    void* lock_buf = nullptr;
    float* staging = nullptr;  // device f32 image of one arena in the reference layout
    size_t staging_len = 0;
    size_t show_smem = 0;    // plain showdown kernel (f64 scratch)
    size_t act_smem = 0;     // fused up-action dynamic smem
    size_t warp_smem = 0;    // warp up-action dynamic smem (one staged reach per warp)
    size_t st_mine_smem = 0, st_opp_smem = 0, st_down_smem = 0;  // staged kernels
    SNode* snodes = nullptr;                   // staged node records (same order as act)
    size_t show_pair_smem = 0;                                    // batched showdowns
    // river programs (cfr_river.cuh): each river betting round solved by one
    // CTA; the level sweeps then cover only the nodes outside river rounds
    bool river = false;
    bool levels_only = false;  // set while a query needs every node's slots (level sweeps everywhere)
    RTree* rtrees = nullptr;
    RStep* rsteps = nullptr;
    int ntrees = 0;
    RLayout rl[2]{};     // per traverser
    int river_grid = 0;  // persistent CTAs (one per SM)
    bool use_river() const { return river && !levels_only; }
    size_t chance_smem = 0;  // runout chance dynamic smem
    cudaGraphExec_t g_iter = nullptr;
    cudaGraphExec_t g_eval[2] = {nullptr, nullptr};
    double* h_dot = nullptr;  // pinned

    // Two pinned chunks for large device -> pageable host copies (allocated
    // on first use): the DMA of one chunk overlaps the spread copy of the
    // other into place, so a copy runs near the pinned rate instead of the
    // pageable one.
    static constexpr size_t kD2HChunk = size_t(64) << 20;  // bytes
    unsigned char* d2h_pin[2] = {nullptr, nullptr};
    cudaEvent_t d2h_ev[2] = {nullptr, nullptr};
    void d2h_large(void* dst, const void* src, size_t bytes) {
        if (bytes < 2 * kD2HChunk) {
            CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            return;
        }
        for (int b = 0; b < 2; b++)
            if (!d2h_pin[b]) {
                CK(cudaMallocHost(&d2h_pin[b], kD2HChunk));
                CK(cudaEventCreateWithFlags(&d2h_ev[b], cudaEventDisableTiming));
            }
        const size_t nc = (bytes + kD2HChunk - 1) / kD2HChunk;
        auto issue = [&](size_t j) {
            const size_t off = j * kD2HChunk, cnt = std::min(kD2HChunk, bytes - off);
            CK(cudaMemcpyAsync(d2h_pin[j & 1], (const unsigned char*)src + off, cnt, cudaMemcpyDeviceToHost, stream));
            CK(cudaEventRecord(d2h_ev[j & 1], stream));
        };
        const unsigned hw = std::thread::hardware_concurrency();
        const int nt = (int)std::max(1u, std::min(8u, hw ? hw : 1u));
        issue(0);
        for (size_t j = 0; j < nc; j++) {
            if (j + 1 < nc) issue(j + 1);  // its buffer's previous chunk was copied out last round
            CK(cudaEventSynchronize(d2h_ev[j & 1]));
            const size_t off = j * kD2HChunk, cnt = std::min(kD2HChunk, bytes - off);
            const unsigned char* from = d2h_pin[j & 1];
            unsigned char* to = (unsigned char*)dst + off;
            const size_t part = (cnt + nt - 1) / nt;
            std::vector<std::thread> ts;
            for (int w = 1; w < nt; w++) {
                const size_t a = std::min(cnt, w * part), e = std::min(cnt, a + part);
                if (a < e) ts.emplace_back([=] { std::memcpy(to + a, from + a, e - a); });
            }
            std::memcpy(to, from, std::min(cnt, part));
            for (auto& t : ts) t.join();
        }
        CK(cudaStreamSynchronize(stream));
    }
    ~EngineImpl() {
        if (stream) cudaStreamSynchronize(stream);
        for (int b = 0; b < 2; b++) {
            if (d2h_ev[b]) cudaEventDestroy(d2h_ev[b]);
            if (d2h_pin[b]) cudaFreeHost(d2h_pin[b]);
        }
        if (g_iter) cudaGraphExecDestroy(g_iter);
        for (auto& g : g_eval)
            if (g) cudaGraphExecDestroy(g);
        if (lock_buf) cudaFree(lock_buf);
        for (void* p : owned) cudaFree(p);
        if (h_dot) cudaFreeHost(h_dot);
        for (cudaEvent_t e : ev_term) cudaEventDestroy(e);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }

    // The f32 reference-layout image in `staging` into device arena `which` of
    // player q (encoded for 16-bit and FP8 arenas, with per-node scales).
    void encode_staging(int which, int q) {
        const unsigned nb = (unsigned)plan.n_anodes[q];
        if (!nb) return;
        const int nh = plan.nh[q];
        void* dst = which == kRegrets ? ar.reg[q] : which == kStrategy ? ar.str[q] : ar.pred[q];
        if (fmt == kFmtF32) {
            k_to_dev<float><<<nb, kThreads, 0, stream>>>(staging, (float*)dst, xnodes[q], nh);
        } else {
            float* dsc = which == kRegrets ? ar.rscale[q] : which == kStrategy ? ar.sscale[q] : ar.pscale[q];
            if (fmt == kFmtFP8)
                k_encode_fp8<<<nb, kThreads, 0, stream>>>(staging, (uint8_t*)dst, dsc, xnodes[q], nh, which == kStrategy);
            else
                k_encode<<<nb, kThreads, 0, stream>>>(staging, dst, dsc, xnodes[q], nh, which == kStrategy);
        }
        CK(cudaGetLastError());
    }
    void upload_locks(const HostSolver& host) {
        if (lock_buf) {
            CK(cudaStreamSynchronize(stream));
            CK(cudaFree(lock_buf));
            lock_buf = nullptr;
        }
        std::vector<long long> off[2];
        std::vector<float> sig;
        for (int p = 0; p < 2; p++) off[p].assign(std::max<uint64_t>(plan.n_anodes[p], 1), -1);
        for (auto& kv : host.locks) {
            const int32_t s = plan.node_sidx[kv.first];
            if (s < 0) continue;  // lock on a branch the device does not traverse
            off[spot->tree.player[kv.first]][s] = (long long)sig.size();
            sig.insert(sig.end(), kv.second.begin(), kv.second.end());
        }
        if (sig.empty()) sig.push_back(0.0f);
        const size_t b0 = off[0].size() * 8, b1 = off[1].size() * 8, bs = sig.size() * 4;
        CK(cudaMalloc(&lock_buf, b0 + b1 + bs));
        char* base = (char*)lock_buf;
        CK(cudaMemcpy(base, off[0].data(), b0, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(base + b0, off[1].data(), b1, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(base + b0 + b1, sig.data(), bs, cudaMemcpyHostToDevice));
        d.lock_off[0] = (const long long*)base;
        d.lock_off[1] = (const long long*)(base + b0);
        d.lock_sig = (const float*)(base + b0 + b1);
        drop_graphs();
        reach_valid = false;
    }
    void drop_graphs() {
        if (g_iter) { cudaGraphExecDestroy(g_iter); g_iter = nullptr; }
        for (auto& g : g_eval)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    // A launch's configuration error (resources, shared memory) is reported
    // at the launch, naming its kind, instead of surfacing later as an
    // invalidated stream capture.
    void launch_ok(int kind) const {
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            throw Error(std::string("cuda: ") + cudaGetErrorString(e) + " launching a " + kKernelNames[kind] +
                        " kernel (dynamic shared memory: showdowns " + std::to_string(show_pair_smem) + " B, up " +
                        std::to_string(st_mine_smem) + "/" + std::to_string(st_opp_smem) + " B, down " +
                        std::to_string(st_down_smem) + " B)");
    }
    template <class F>
    void timed(Profile* pr, int kind, F launch) {
        if (!pr) {
            launch();
            launch_ok(kind);
            return;
        }
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        CK(cudaEventRecord(a, stream));
        launch();
        CK(cudaEventRecord(b, stream));
        CK(cudaEventSynchronize(b));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, a, b));
        pr->ms[kind] += ms;
        pr->launches[kind] += 1;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }

    template <int FMT, int KA, class TT>
    void up_action_t(const Span& sa, int p, int eval) {
        const ActItem* it = act + sa.start;
        if (eval < 0) k_up_action<FMT, 0, KA, TT><<<sa.count, kThreads, act_smem, stream>>>(d, ar, it, p, 0);
        else k_up_action<FMT, 1, KA, TT><<<sa.count, kThreads, act_smem, stream>>>(d, ar, it, p, eval);
    }
    template <int FMT, int KA>
    void up_action(const Span& sa, int p, int eval) {
        if (term64) up_action_t<FMT, KA, long long>(sa, p, eval);
        else up_action_t<FMT, KA, float>(sa, p, eval);
    }
    template <int FMT, int KA, class TT>
    static void set_up_smem(size_t bytes) {
        set_smem((const void*)k_up_action<FMT, 0, KA, TT>, bytes);
        set_smem((const void*)k_up_action<FMT, 1, KA, TT>, bytes);
    }
    template <int FMT, int KA>
    void down_action(const Span& sa, int mode) {
        if (staged) {
            ks_down<FMT><<<sa.count, kSThreads, st_down_smem, stream>>>(d, ar, snodes + sa.start, mode);
        } else if (warp) {
            const unsigned grid = (sa.count + kWarps - 1) / kWarps;
            kw_down_action<FMT, KA><<<grid, kThreads, 0, stream>>>(d, ar, act + sa.start, (int)sa.count, mode);
        } else {
            k_down_action<FMT, KA><<<sa.count, kThreads, 0, stream>>>(d, ar, act + sa.start, mode);
        }
    }
    template <int FMT, int KA>
    void warp_up_action(const Span& sa, int p, int eval) {
        const unsigned grid = (sa.count + kWarps - 1) / kWarps;
        const ActItem* it = act + sa.start;
        if (eval < 0) kw_up_action<FMT, 0, KA><<<grid, kThreads, warp_smem, stream>>>(d, ar, it, (int)sa.count, p, 0);
        else kw_up_action<FMT, 1, KA><<<grid, kThreads, warp_smem, stream>>>(d, ar, it, (int)sa.count, p, eval);
    }
    template <int FMT, int KA>
    static void set_warp_smem(size_t bytes) {
        set_smem((const void*)kw_up_action<FMT, 0, KA>, bytes);
        set_smem((const void*)kw_up_action<FMT, 1, KA>, bytes);
    }
    template <int FMT, bool MINE>
    void staged_up(const Span& s, int p, int eval) {
        if (!s.count) return;
        const SNode* it = snodes + s.start;
        const size_t sm = MINE ? st_mine_smem : st_opp_smem;
        if (eval < 0) ks_up<FMT, 0, MINE><<<s.count, kSThreads, sm, stream>>>(d, ar, it, p, 0);
        else ks_up<FMT, 1, MINE><<<s.count, kSThreads, sm, stream>>>(d, ar, it, p, eval);
    }
    template <int FMT>
    static void set_staged_smem(size_t mine, size_t opp) {
        set_smem((const void*)ks_up<FMT, 0, true>, mine);
        set_smem((const void*)ks_up<FMT, 1, true>, mine);
        set_smem((const void*)ks_up<FMT, 0, false>, opp);
        set_smem((const void*)ks_up<FMT, 1, false>, opp);
    }
    // Up sweep of one level's action nodes.  The staged engine launches the
    // traverser's nodes and the opponent's separately (each launch's kernel is
    // specialised for its side and sized for its shared memory).
    // The action nodes of level l the level sweeps cover: all of them, or,
    // with river programs, those outside river betting rounds.
    Span act_level(int l, int actor) const {
        return use_river() ? plan.act_span_upper[actor][l] : plan.act_span_actor[actor][l];
    }
    void launch_up_level(int l, int p, int eval) {
        if (staged) {
            const Span mine = act_level(l, p), opp = act_level(l, 1 - p);
            if (fmt == kFmtF32) {
                staged_up<kDevF32, true>(mine, p, eval);
                staged_up<kDevF32, false>(opp, p, eval);
            } else if (fmt == kFmtFP8) {
                staged_up<kDevFP8, true>(mine, p, eval);
                staged_up<kDevFP8, false>(opp, p, eval);
            } else {
                staged_up<kDevI16, true>(mine, p, eval);
                staged_up<kDevI16, false>(opp, p, eval);
            }
            return;
        }
        launch_up_action(plan.act_span[l], p, eval);
    }
    void launch_up_action(const Span& sa, int p, int eval) {
        if (warp) {
            if (fmt == kFmtF32) {
                if (wide) warp_up_action<kDevF32, 32>(sa, p, eval);
                else warp_up_action<kDevF32, 8>(sa, p, eval);
            } else {
                if (wide) warp_up_action<kDevI16, 32>(sa, p, eval);
                else warp_up_action<kDevI16, 8>(sa, p, eval);
            }
            return;
        }
        if (fmt == kFmtF32) {
            if (wide) up_action<kDevF32, 32>(sa, p, eval);
            else up_action<kDevF32, 8>(sa, p, eval);
        } else {
            if (wide) up_action<kDevI16, 32>(sa, p, eval);
            else up_action<kDevI16, 8>(sa, p, eval);
        }
    }
    void launch_down_action(const Span& sa, int mode) {
        if (fmt == kFmtFP8) {  // the staged engine only
            ks_down<kDevFP8><<<sa.count, kSThreads, st_down_smem, stream>>>(d, ar, snodes + sa.start, mode);
            return;
        }
        if (fmt == kFmtF32) {
            if (wide) down_action<kDevF32, 32>(sa, mode);
            else down_action<kDevF32, 8>(sa, mode);
        } else {
            if (wide) down_action<kDevI16, 32>(sa, mode);
            else down_action<kDevI16, 8>(sa, mode);
        }
    }

    void launch_chance(const Span& sc, int p) {
        // runout showdowns: f32 sums in the fused engine, f64 in the plain one
        if (plan.fused && !term64) k_chance<float><<<sc.count, kThreads, chance_smem, stream>>>(d, chance + sc.start, p);
        else k_chance<long long><<<sc.count, kThreads, chance_smem, stream>>>(d, chance + sc.start, p);
    }

    // Down sweep.  qmask: the players whose reach vectors are recomputed.  In a
    // CFR iteration only the opponent's are: the traverser's own reach depends
    // on its own strategy only, which has not changed since the previous
    // sweep computed it (that sweep's traverser was the other player), so its
    // slots still hold exactly the values a full recomputation would write.
    void down(int qmask, int mode, Profile* pr) {
        timed(pr, 0, [&] { k_copy_root<<<4, kThreads, 0, stream>>>(d); });
        const int L = plan.num_levels;
        for (int l = 0; l < L; l++) {
            if (use_river()) {  // two runs when both players' reach is refreshed
                for (int q = 0; q < 2; q++) {
                    const Span sq = act_level(l, q);
                    if ((qmask >> q & 1) && sq.count) timed(pr, 1, [&] { launch_down_action(sq, mode); });
                }
            } else {
                const Span sa = qmask == 3 ? plan.act_span[l] : plan.act_span_actor[qmask == 1 ? 0 : 1][l];
                if (sa.count) timed(pr, 1, [&] { launch_down_action(sa, mode); });
            }
            const Span se = plan.edge_span[l];
            if (se.count)
                timed(pr, 2, [&] { k_down_chance<<<se.count, kThreads, 0, stream>>>(d, edge + se.start, qmask); });
        }
    }
    // Before the first CFR sweep after anything else wrote the reach slots
    // (engine start, eval sweeps, lock changes): both players' reach.
    void prime() {
        if (reach_valid) return;
        down(3, 0, nullptr);
        CK(cudaGetLastError());
        reach_valid = true;
    }
    // One sweep for traverser p.  eval < 0: CFR iteration; 0/1: BR / average.
    void sweep(int p, int eval, Profile* pr) {
        const int L = plan.num_levels;
        if (eval < 0) {
            down(1 << (1 - p), 0, pr);
        } else {
            down(3, 1, pr);
            reach_valid = false;
        }
        // depth-limited: the turn leaves' values from the network, before
        // any level of the up sweep reads them
        if (leaf) leaf->run(p, d.reach[0], (size_t)d.rstr[0], d.reach[1], (size_t)d.rstr[1], d.cfv, (size_t)d.nh_max, stream);
        // every river betting round at once, before any level of the up sweep
        // reads a round's root value (counted with the up sweep's action kind)
        if (use_river()) timed(pr, 6, [&] { launch_river(p, eval); });
        // Terminal kernels (folds and showdowns with slots of their own) read
        // only reach vectors, so in a captured sweep they run on a second
        // stream, every level of them, beside the chain of chance and action
        // levels; the chain waits for level l + 1's terminals before it
        // consumes them at level l.
        const bool fork = pr == nullptr && side != nullptr;
        if (fork) {
            CK(cudaEventRecord(ev_fork, stream));
            CK(cudaStreamWaitEvent(side, ev_fork, 0));
            for (int l = L - 1; l >= 0; l--) {
                launch_terminals(l, p, side, nullptr);
                CK(cudaEventRecord(ev_term[l], side));
            }
        }
        for (int l = L - 1; l >= 0; l--) {
            if (!fork) launch_terminals(l, p, stream, pr);
            else if (l + 1 < L) CK(cudaStreamWaitEvent(stream, ev_term[l + 1], 0));
            reduce_level(l, p);  // a shard: the children of this level's top chance nodes from every shard
            const Span sc = plan.chance_span[l];
            if (sc.count) timed(pr, 5, [&] { launch_chance(sc, p); });
            const bool any = use_river() ? act_level(l, 0).count + act_level(l, 1).count > 0 : plan.act_span[l].count > 0;
            if (any) timed(pr, 6, [&] { launch_up_level(l, p, eval); });
        }
        if (fork) {
            CK(cudaEventRecord(ev_join, side));
            CK(cudaStreamWaitEvent(stream, ev_join, 0));
        }
        CK(cudaGetLastError());
    }
    template <int FMT>
    void launch_river_t(int p, int eval) {
        const RLayout& L = rl[p];
        const int ms = (int)plan.max_sorted;
        if (eval < 0)
            kr_river<FMT, 0, kRiverNT><<<river_grid, kRiverNT, L.total, stream>>>(d, ar, rtrees, rsteps, ntrees, p, 0,
                                                                               ms, L);
        else
            kr_river<FMT, 1, kRiverNT><<<river_grid, kRiverNT, L.total, stream>>>(d, ar, rtrees, rsteps, ntrees, p,
                                                                               eval, ms, L);
    }
    void launch_river(int p, int eval) {
        if (fmt == kFmtF32) launch_river_t<kDevF32>(p, eval);
        else if (fmt == kFmtFP8) launch_river_t<kDevFP8>(p, eval);
        else launch_river_t<kDevI16>(p, eval);
    }
    void launch_terminals(int l, int p, cudaStream_t st, Profile* pr) {
        const Span sf = plan.fold_span[l];
        if (sf.count) timed(pr, 3, [&] { k_fold<<<sf.count, kThreads, 0, st>>>(d, fold + sf.start, p); });
        const Span ss = plan.show_span[l];
        const Span sb = use_river() ? plan.show_batch_span_upper[l] : plan.show_batch_span[l];
        if (staged ? sb.count > 0 : ss.count > 0)
            timed(pr, 4, [&] {
                if (staged) {
                    if (plan.max_sorted > 384)
                        ks_show_pair<256><<<sb.count, 256, show_pair_smem, st>>>(d, show, show_batch + sb.start, p,
                                                                                  (int)plan.max_sorted);
                    else
                        ks_show_pair<128><<<sb.count, 128, show_pair_smem, st>>>(d, show, show_batch + sb.start, p,
                                                                                  (int)plan.max_sorted);
                } else {
                    k_showdown<<<ss.count, kThreads, show_smem, st>>>(d, show + ss.start, p);
                }
            });
    }
    void record_iteration() {
        k_begin_iteration<<<1, 1, 0, stream>>>(d.iter, d.disc, algo);
        sweep(0, -1, nullptr);
        sweep(1, -1, nullptr);
    }
    void record_eval(int mode) {
        for (int p = 0; p < 2; p++) {
            sweep(p, mode, nullptr);
            k_root_dot<<<1, kThreads, 0, stream>>>(d, p, p);
        }
        CK(cudaMemcpyAsync(h_dot, d.dot, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    }
    // Device error bits (bounded waits that gave up): read at every
    // synchronisation point; reported once, then cleared.
    void check_err() {
        unsigned e = 0;
        CK(cudaMemcpyAsync(&e, d.err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
        if (leaf) {
            unsigned ne = 0;
            CK(cudaMemcpyAsync(&ne, leaf->net().err_word(), sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            if (ne) {
                CK(cudaMemsetAsync(leaf->net().err_word(), 0, sizeof(unsigned), stream));
                CK(cudaStreamSynchronize(stream));
                throw Error("timeout: a tensor-core matrix product's wait gave up");
            }
        }
        CK(cudaStreamSynchronize(stream));
        if (e) {
            CK(cudaMemsetAsync(d.err, 0, sizeof(unsigned), stream));
            CK(cudaStreamSynchronize(stream));
            throw Error(std::string("timeout: ") + ((e & 1u) ? "a staged copy did not complete within its wait limit"
                                                              : "a staged copy was refused (misaligned)"));
        }
    }
    cudaGraphExec_t capture(int which) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            if (which < 0) record_iteration();
            else record_eval(which);
        } catch (...) {
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        CK(cudaStreamEndCapture(stream, &g));
        if (which < 0) {  // the kernels one iteration launches: the graph's kernel nodes
            size_t nn = 0;
            CK(cudaGraphGetNodes(g, nullptr, &nn));
            std::vector<cudaGraphNode_t> nodes(nn);
            if (nn) CK(cudaGraphGetNodes(g, nodes.data(), &nn));
            uint32_t k = 0;
            for (auto nd : nodes) {
                cudaGraphNodeType ty;
                CK(cudaGraphNodeGetType(nd, &ty));
                k += ty == cudaGraphNodeTypeKernel;
            }
            iter_kernels = k;
        }
        cudaGraphExec_t ex;
        CK(cudaGraphInstantiate(&ex, g, 0));
        cudaGraphDestroy(g);
        return ex;
    }
    uint32_t iter_kernels = 0;  // kernel nodes of the captured iteration graph
    std::unique_ptr<LeafEvaluator> leaf;  // depth-limited solves: the turn leaves' network
    std::shared_ptr<ShardReducer> reducer;  // sharded spot: sums the top chance nodes over the shards
    bool uncaptured = false;                // the reducer syncs on the host: plain launches, no graphs
    // the values of the level's top chance nodes' children, summed over the
    // shards (one shard holds each, the others hold zeros)
    void reduce_level(int l, int p) {
        (void)p;
        if (!reducer || l >= (int)plan.reduce_span.size() || !plan.reduce_span[l].count) return;
        // another shard's children hold the previous sum here: zero them so
        // that the sum adds each child's value to zeros only
        const Span r = plan.reduce_span[l], o = plan.own_span[l];
        const size_t w = d.nh_max;
        if (o.start > r.start) CK(cudaMemsetAsync(d.cfv + (size_t)r.start * w, 0, (size_t)(o.start - r.start) * w * 4, stream));
        const uint32_t oe = o.start + o.count, re = r.start + r.count;
        if (re > oe) CK(cudaMemsetAsync(d.cfv + (size_t)oe * w, 0, (size_t)(re - oe) * w * 4, stream));
        reducer->reduce(d.cfv + (size_t)r.start * w, (size_t)r.count * w, stream);
    }
};


// River programs (cfr_river.cuh): the subtree list and steps, each river
// board's showdown table image per player, the kernel's shared-memory layout
// per traverser and its grid.  E.river stays false when the layout does not
// fit the device's shared memory.
template <int FMT>
static void river_smem_attrs(size_t bytes) {
    set_smem((const void*)kr_river<FMT, 0, kRiverNT>, bytes);
    set_smem((const void*)kr_river<FMT, 1, kRiverNT>, bytes);
}
static void setup_river(EngineImpl& E, const Spot& sp) {
    const Plan& P = E.plan;
    if (!P.river || P.rtrees.empty()) return;
    int dev = 0, optin = 0, nsm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, (const void*)kr_river<kDevI16, 0, kRiverNT>));
    const int esz = fmt_bytes(E.fmt == kFmtF32 ? kDevF32 : E.fmt == kFmtFP8 ? kDevFP8 : kDevI16);
    const int depth = P.river_depth + 1;
    int nslot = 6;
    size_t need = 0;
    for (; nslot >= 2; nslot--) {
        need = 0;
        for (int p = 0; p < 2; p++) {
            E.rl[p] = river_layout(E.d.nh_pad, esz, E.pcfr, depth, p, (int)P.max_sorted, nslot);
            need = std::max<size_t>(need, E.rl[p].total);
        }
        if (need + fa.sharedSizeBytes <= (size_t)optin) break;
    }
    if (nslot < 2) return;  // the level sweeps keep the river
    auto& O = E.owned;
    size_t& B = E.bytes;
    E.rtrees = dupload(P.rtrees, O, &B);
    E.rsteps = dupload(P.rsteps, O, &B);
    E.ntrees = (int)P.rtrees.size();
    const uint32_t msort = P.max_sorted;
    for (int o = 0; o < 2; o++) {
        std::vector<uint32_t> img, off;
        for (uint32_t sl = 0; sl < P.num_slots; sl++) {
            off.push_back((uint32_t)img.size());
            const uint32_t m = P.sorted_cnt[o][sl], soff = P.sorted_off[o][sl];
            const uint32_t* co = P.ccard_off[o].data() + (size_t)sl * 53;
            const uint32_t c0 = co[0], ne = co[52] - c0;
            const size_t base = img.size();
            img.resize(base + river_tab_words((int)m, (int)ne), 0u);
            for (int c = 0; c < 53; c++) img[base + c] = co[c] - c0;
            uint32_t* ent = img.data() + base + 56;
            for (uint32_t f = 0; f < m + ne; f++) {
                uint32_t h, head, oi;
                if (f < m) {
                    h = P.sorted_idx[o][soff + f];
                    head = f == 0;
                    oi = f + 1;
                } else {
                    const uint32_t t = f - m, c = P.ccard_card[o][c0 + t];
                    h = P.sorted_idx[o][soff + P.ccard_pos[o][c0 + t]];
                    head = t == 0 || P.ccard_card[o][c0 + t - 1] != c;
                    oi = msort + 2 + t + c;
                }
                if (h > 0xFFFu || oi > 0xFFFFu) return;  // beyond the packed entry's fields: keep the level sweeps
                ent[f] = h | head << 12 | oi << 16;
            }
        }
        off.push_back((uint32_t)img.size());
        E.d.rtab[o] = dupload(img, O, &B);
        E.d.rtab_off[o] = dupload(off, O, &B);
    }
    river_smem_attrs<kDevF32>(need);
    river_smem_attrs<kDevI16>(need);
    river_smem_attrs<kDevFP8>(need);
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kr_river<kDevI16, 0, kRiverNT>, kRiverNT, need));
    if (per_sm < 1) return;
    E.river_grid = std::min(per_sm * nsm, E.ntrees);
    E.river = true;
}

// --------------------------------------------------------------- GpuEngine
GpuEngine::GpuEngine(const HostSolver& host, int fmt, int engine) : GpuEngine(host, fmt, engine, 0, 1, nullptr) {}

GpuEngine::GpuEngine(const HostSolver& host, int fmt, int engine, int shard, int nshards,
                     std::shared_ptr<ShardReducer> reducer, std::shared_ptr<LeafNet> leaf_net)
    : d_(new EngineImpl()) {
    EngineImpl& E = *d_;
    if (leaf_net && nshards > 1) throw Error("invalid argument: a depth-limited solve runs on one shard");
    if (nshards > 1 && !reducer) throw Error("invalid argument: a sharded engine needs a reducer");
    E.reducer = nshards > 1 ? reducer : nullptr;
    E.uncaptured = E.reducer && !E.reducer->capturable();
    const Spot& sp = *host.spot;
    g_uploaded = 0;
    if (engine < kEngineFused || engine > kEngineStagedRiver) throw Error("unknown engine kind");
    const bool staged_kind = engine == kEngineStaged || engine == kEngineStagedRiver;
    const int fuse = engine == kEnginePlain                        ? kFuseNone
                     : (engine == kEngineWarp || staged_kind)      ? kFuseFolds
                                                                   : kFuseAll;
    E.warp = engine == kEngineWarp || staged_kind;  // staged falls back to warp kernels
    E.term64 = engine != kEngineFused32;
    E.spot = &sp;
    E.algo = host.algo;
    E.pcfr = host.algo == kPcfrPlus;
    if (fmt == kFmtI16SR) {  // 16-bit arenas, stochastic rounding in the update
        E.ar.sr = 1;
        fmt = kFmtI16;
    }
    E.fmt = fmt < 0 ? (host.storage == kStoreF32 ? kFmtF32 : kFmtI16) : fmt;
    if (E.fmt != kFmtF32 && E.fmt != kFmtI16 && E.fmt != kFmtFP8) throw Error("unknown device arena format");
    if (E.fmt == kFmtFP8 && !staged_kind) throw Error("FP8 arenas run on the staged engine only");
    E.iteration = host.iteration;
    E.plan = build_plan(sp, host.use_iso, fuse, shard, nshards, leaf_net != nullptr,
                        engine == kEngineStagedRiver && !leaf_net);
    const Plan& P = E.plan;
    if (P.max_children > 32u) throw Error("an action node with more than 32 actions is not supported on the GPU");
    E.wide = P.max_children > 8u;
    E.staged = staged_kind && P.max_children <= (uint32_t)kSKA;
    if (E.fmt == kFmtFP8 && !E.staged) throw Error("FP8 arenas need nodes of at most 4 actions (the staged kernels)");
    if (P.nh_max > kThreads * kMaxHpt) throw Error("more than 1536 hands per player is not supported on the GPU");
    CK(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&E.side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&E.ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&E.ev_join, cudaEventDisableTiming));
    E.ev_term.resize(std::max(P.num_levels, 1));
    for (auto& e : E.ev_term) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    size_t& B = E.bytes;
    auto& O = E.owned;
    Dev& d = E.d;
    d.nh[0] = P.nh[0];
    d.nh[1] = P.nh[1];
    d.nh_pad = (P.nh_max + 3) / 4 * 4;
    d.nh_max = d.nh_pad;  // cfv slot stride: 16-byte aligned slots
    d.rstr[0] = (P.nh[0] + 3) / 4 * 4;
    d.rstr[1] = (P.nh[1] + 3) / 4 * 4;
    d.scr_elems = (int)(4 * P.max_sorted + 105);
    uint32_t max_nterm = 0;
    bool runouts = false;
    for (auto& a : P.act) max_nterm = std::max(max_nterm, a.nterm);
    for (auto& c : P.chance) runouts = runouts || c.nterm > 0;
    d.max_nterm = (int)max_nterm;
    for (int q = 0; q < 2; q++) {
        const Hands& h = sp.hands[q];
        d.c1[q] = dupload(h.c1, O, &B);
        d.c2[q] = dupload(h.c2, O, &B);
        d.mask[q] = dupload(h.mask, O, &B);
        d.same[q] = dupload(sp.same[q], O, &B);
        d.w[q] = dupload(h.w, O, &B);
        std::vector<uint16_t> hp;
        for (auto& t : sp.hand_perm[q]) hp.insert(hp.end(), t.begin(), t.end());
        d.hperm[q] = dupload(hp, O, &B);
        d.hcard_off[q] = dupload(P.hcard_off[q], O, &B);
        d.hcard_idx[q] = dupload(P.hcard_idx[q], O, &B);
        d.sorted_off[q] = dupload(P.sorted_off[q], O, &B);
        d.sorted_cnt[q] = dupload(P.sorted_cnt[q], O, &B);
        d.sorted_idx[q] = dupload(P.sorted_idx[q], O, &B);
        d.ccard_off[q] = dupload(P.ccard_off[q], O, &B);
        d.ccard_pos[q] = dupload(P.ccard_pos[q], O, &B);
        d.ccard_card[q] = dupload(P.ccard_card[q], O, &B);
        d.bin_off[q] = dupload(P.bin_off[q], O, &B);
        d.bin_start[q] = dupload(P.bin_start[q], O, &B);
        d.rank_off[q] = dupload(P.rank_off[q], O, &B);
        d.rank_cnt[q] = dupload(P.rank_cnt[q], O, &B);
        d.rank[q] = dupload(P.rank[q], O, &B);
        d.zero_off[q] = dupload(P.zero_off[q], O, &B);
        d.zero_idx[q] = dupload(P.zero_idx[q], O, &B);
        d.reach[q] = (float*)dalloc(P.n_rslots[q] * (size_t)d.rstr[q] * sizeof(float), O, &B);
        d.node_id[q] = dupload(P.anode_id[q], O, &B);
    }
    d.cards = dupload(P.cards, O, &B);
    d.crefs = dupload(P.crefs, O, &B);
    d.terms = dupload(P.terms, O, &B);
    d.cfv = (float*)dalloc(P.n_cslots * (size_t)d.nh_max * sizeof(float), O, &B);
    d.disc = (float*)dalloc(4 * sizeof(float), O, &B);
    d.iter = (unsigned*)dalloc(sizeof(unsigned), O, &B);
    d.dot = (double*)dalloc(4 * sizeof(double), O, &B);
    d.err = (unsigned*)dalloc(sizeof(unsigned), O, &B);
    CK(cudaMemcpy(d.iter, &E.iteration, sizeof(unsigned), cudaMemcpyHostToDevice));
    E.act = dupload(P.act, O, &B);
    E.edge = dupload(P.edge, O, &B);
    E.fold = dupload(P.fold, O, &B);
    E.show = dupload(P.show, O, &B);
    E.show_batch = dupload(P.show_batch, O, &B);
    E.chance = dupload(P.chance, O, &B);
    const size_t tsz = E.term64 ? sizeof(double) : sizeof(float);
    E.show_smem = (size_t)d.scr_elems * sizeof(double);
    if (E.warp) E.warp_smem = (size_t)kWarps * d.nh_pad * sizeof(float);
    if (E.staged) {
        // node records, packed hand words, fixed-stride card lists
        PodVec<SNode> sn(P.act.size());
        parallel_for((P.act.size() + 65535) / 65536, [&](size_t chunk) {
          for (size_t k = chunk * 65536; k < std::min(P.act.size(), (chunk + 1) * 65536); k++) {
            const ActItem& a = P.act[k];
            SNode& x = sn[k];
            std::memset(&x, 0, sizeof(x));
            x.aoff = a.aoff;
            x.cslot = a.cslot;
            x.rslot = a.rslot;
            x.oslot = a.oslot;
            x.sidx = a.sidx;
            x.actor = a.actor;
            x.na = a.na;
            x.fk = kNoSlot;
            for (uint32_t c = 0; c < (uint32_t)kSKA; c++) {
                x.cs[c] = kNoSlot;
                x.rs[c] = kNoSlot;
                if (c >= a.na) continue;
                const ChildRef& r = P.crefs[a.cref + c];
                x.cs[c] = r.cslot;
                x.rs[c] = r.rslot;
                if (r.kind == kChildFold) {
                    const TermInfo& t = P.terms[r.term];
                    x.fk = c;
                    x.folder = t.aux;
                    x.twin = t.twin;
                    x.tlose = t.tlose;
                }
            }
          }
        });
        E.snodes = dupload(sn, O, &B);
        for (int q = 0; q < 2; q++) {
            const Hands& h = sp.hands[q];
            std::vector<uint32_t> hi(h.c1.size());
            for (size_t i = 0; i < hi.size(); i++) {
                const uint32_t s = sp.same[q][i];
                hi[i] = (uint32_t)h.c1[i] | (uint32_t)h.c2[i] << 6 | (s == kSentinel ? 0xFFFFu : s) << 16;
            }
            d.hinfo[q] = dupload(hi, O, &B);
            std::vector<uint16_t> h52(52 * 52, 0xFFFF);
            for (int c = 0; c < 52; c++)
                for (uint32_t k = P.hcard_off[q][c], j = 0; k < P.hcard_off[q][c + 1]; k++, j++) h52[c * 52 + j] = P.hcard_idx[q][k];
            d.hcard52[q] = dupload(h52, O, &B);
        }
        const int esz = fmt_bytes(E.fmt);
        E.st_mine_smem = SLayout(d.nh_pad, esz, E.pcfr, kSUpMine).total;
        E.st_opp_smem = SLayout(d.nh_pad, esz, E.pcfr, kSUpOpp).total;
        E.st_down_smem = SLayout(d.nh_pad, esz, E.pcfr, kSDown).total;
        EngineImpl::set_staged_smem<kDevF32>(E.st_mine_smem, E.st_opp_smem);
        EngineImpl::set_staged_smem<kDevI16>(E.st_mine_smem, E.st_opp_smem);
        EngineImpl::set_staged_smem<kDevFP8>(E.st_mine_smem, E.st_opp_smem);
        set_smem((const void*)ks_down<kDevF32>, E.st_down_smem);
        set_smem((const void*)ks_down<kDevI16>, E.st_down_smem);
        set_smem((const void*)ks_down<kDevFP8>, E.st_down_smem);
        E.show_pair_smem = show_pair_smem_bytes(d.nh_pad, (int)P.max_sorted);
        set_smem((const void*)ks_show_pair<128>, E.show_pair_smem);
        set_smem((const void*)ks_show_pair<256>, E.show_pair_smem);
        const std::pair<const void*, int> show_fns[2] = {{(const void*)ks_show_pair<128>, 128},
                                                         {(const void*)ks_show_pair<256>, 256}};
        for (const auto& fn_nt : show_fns) {
            cudaFuncAttributes fa;
            CK(cudaFuncGetAttributes(&fa, fn_nt.first));
            if ((size_t)fa.maxDynamicSharedSizeBytes < E.show_pair_smem || fa.maxThreadsPerBlock < fn_nt.second)
                throw Error("showdown kernel limits: " + std::to_string(fa.maxDynamicSharedSizeBytes) +
                            " B dynamic shared memory (needs " + std::to_string(E.show_pair_smem) + "), " +
                            std::to_string(fa.maxThreadsPerBlock) + " threads, " + std::to_string(fa.numRegs) +
                            " registers, " + std::to_string(fa.sharedSizeBytes) + " B static");
        }
        setup_river(E, sp);
    }
    if (max_nterm && !E.warp) E.act_smem = (size_t)d.scr_elems * tsz + 2 * (size_t)max_nterm * d.nh_pad * sizeof(float);
    if (runouts) E.chance_smem = (size_t)d.scr_elems * tsz + 2 * (size_t)d.nh_pad * sizeof(float);
    set_smem((const void*)k_showdown, E.show_smem);
    set_smem((const void*)k_chance<float>, E.chance_smem);
    set_smem((const void*)k_chance<long long>, E.chance_smem);
    EngineImpl::set_up_smem<kDevF32, 8, float>(E.act_smem);
    EngineImpl::set_up_smem<kDevI16, 8, float>(E.act_smem);
    EngineImpl::set_up_smem<kDevF32, 32, float>(E.act_smem);
    EngineImpl::set_up_smem<kDevI16, 32, float>(E.act_smem);
    EngineImpl::set_up_smem<kDevF32, 8, long long>(E.act_smem);
    EngineImpl::set_up_smem<kDevI16, 8, long long>(E.act_smem);
    EngineImpl::set_up_smem<kDevF32, 32, long long>(E.act_smem);
    EngineImpl::set_up_smem<kDevI16, 32, long long>(E.act_smem);
    EngineImpl::set_warp_smem<kDevF32, 8>(E.warp_smem);
    EngineImpl::set_warp_smem<kDevI16, 8>(E.warp_smem);
    EngineImpl::set_warp_smem<kDevF32, 32>(E.warp_smem);
    EngineImpl::set_warp_smem<kDevI16, 32>(E.warp_smem);

    // arenas
    const size_t esz = (size_t)fmt_bytes(E.fmt);
    for (int q = 0; q < 2; q++) {
        const size_t len = P.arena_len[q];
        E.ar.reg[q] = dalloc(len * esz, O, &B);
        E.ar.str[q] = dalloc(len * esz, O, &B);
        E.ar.pred[q] = E.pcfr ? dalloc(len * esz, O, &B) : nullptr;
        if (E.fmt != kFmtF32) {
            E.ar.rscale[q] = (float*)dalloc(std::max<uint64_t>(P.n_anodes[q], 1) * 4, O, &B);
            E.ar.sscale[q] = (float*)dalloc(std::max<uint64_t>(P.n_anodes[q], 1) * 4, O, &B);
            E.ar.pscale[q] = E.pcfr ? (float*)dalloc(std::max<uint64_t>(P.n_anodes[q], 1) * 4, O, &B) : nullptr;
        }
        for (uint64_t s = 0; s < P.n_anodes[q]; s++) {
            const uint32_t nd = P.anode_id[q][s];
            E.hx[q].push_back({sp.tree.data_off[nd], P.anode_off[q][s], sp.tree.nchild[nd], (uint32_t)s});
        }
        E.xnodes[q] = dupload(E.hx[q], O, &B);
    }
    E.staging_len = std::max<uint64_t>(std::max(sp.tree.data_size[0], sp.tree.data_size[1]), 1);
    E.staging = (float*)dalloc(E.staging_len * sizeof(float), O, &B);
    CK(cudaMallocHost(&E.h_dot, 4 * sizeof(double)));

    // upload arenas: quants directly when host and device are both 16-bit, else via f32 (+ encode);
    // nothing to upload while the host arenas are still all zero (so are the device's)
    std::vector<float> img;  // f32 image of one host arena, when one is needed
    for (int q = 0; q < 2 && !host.arenas_zero; q++) {
        const int nh = P.nh[q];
        const unsigned nb = (unsigned)P.n_anodes[q];
        if (!nb) continue;
        for (int which = 0; which < 3; which++) {
            if (which == kPreds && !E.pcfr) continue;
            void* dst = which == kRegrets ? E.ar.reg[q] : which == kStrategy ? E.ar.str[q] : E.ar.pred[q];
            const Arena* ha = which == kRegrets ? &host.regrets[q] : which == kStrategy ? &host.strat[q]
                              : (host.have_preds ? &host.preds[q] : nullptr);
            if (!ha) continue;  // predictions start at zero
            if (E.fmt == kFmtI16 && ha->kind != 0) {
                const size_t len = sp.tree.data_size[q];
                if (ha->kind == 1) CK(cudaMemcpy(E.staging, ha->qi.data(), len * 2, cudaMemcpyHostToDevice));
                else CK(cudaMemcpy(E.staging, ha->qu.data(), len * 2, cudaMemcpyHostToDevice));
                g_uploaded += len * 2 + P.n_anodes[q] * 4;
                k_to_dev<uint16_t><<<nb, kThreads, 0, E.stream>>>((const uint16_t*)E.staging, (uint16_t*)dst, E.xnodes[q], nh);
                std::vector<float> sc(P.n_anodes[q]);
                for (uint64_t s = 0; s < P.n_anodes[q]; s++) sc[s] = ha->scale[P.anode_id[q][s]];
                float* dsc = which == kRegrets ? E.ar.rscale[q] : which == kStrategy ? E.ar.sscale[q] : E.ar.pscale[q];
                CK(cudaMemcpyAsync(dsc, sc.data(), sc.size() * 4, cudaMemcpyHostToDevice, E.stream));
                CK(cudaStreamSynchronize(E.stream));
                continue;
            }
            const float* src32;
            if (ha->kind == 0) {  // f32 host arena: already the image
                src32 = ha->f.data();
            } else {
                img.resize(E.staging_len);
                host.arena_f32(which, q, img.data());
                src32 = img.data();
            }
            CK(cudaMemcpy(E.staging, src32, sp.tree.data_size[q] * 4, cudaMemcpyHostToDevice));
            g_uploaded += sp.tree.data_size[q] * 4;
            E.encode_staging(which, q);
            CK(cudaStreamSynchronize(E.stream));
        }
    }
    E.upload_locks(host);
    if (leaf_net) E.leaf = std::make_unique<LeafEvaluator>(leaf_net, sp, P.leaves);
    CK(cudaStreamSynchronize(E.stream));
    E.uploaded = g_uploaded;
}

GpuEngine::~GpuEngine() = default;
uint64_t GpuEngine::upload_bytes() const { return d_->uploaded; }
uint32_t GpuEngine::river_programs() const { return d_->river ? (uint32_t)d_->ntrees : 0u; }

uint32_t GpuEngine::iteration_kernels() {
    EngineImpl& E = *d_;
    if (E.uncaptured) return 0;  // no graph
    if (!E.g_iter) E.g_iter = E.capture(-1);
    return E.iter_kernels;
}

void GpuEngine::iterate(int n) {
    EngineImpl& E = *d_;
    if (E.uncaptured) {
        for (int k = 0; k < n; k++) {
            E.prime();
            E.record_iteration();
            E.iteration++;
        }
        CK(cudaGetLastError());
        return;
    }
    for (int k = 0; k < n; k++) {
        if (!E.g_iter) E.g_iter = E.capture(-1);
        E.prime();
        CK(cudaGraphLaunch(E.g_iter, E.stream));
        E.iteration++;
    }
    CK(cudaGetLastError());
}

double GpuEngine::time_iterations(int n) {
    EngineImpl& E = *d_;
    if (E.uncaptured) throw Error("time_iterations needs the captured iteration (not an engine of a shard group)");
    if (!E.g_iter) E.g_iter = E.capture(-1);
    E.prime();
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, E.stream));
    for (int k = 0; k < n; k++) {
        CK(cudaGraphLaunch(E.g_iter, E.stream));
        E.iteration++;
    }
    CK(cudaEventRecord(b, E.stream));
    CK(cudaEventSynchronize(b));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    E.check_err();
    return ms;
}

Profile GpuEngine::iterate_profiled() {
    EngineImpl& E = *d_;
    Profile pr;
    std::memset(&pr, 0, sizeof(pr));
    CK(cudaStreamSynchronize(E.stream));
    E.prime();
    k_begin_iteration<<<1, 1, 0, E.stream>>>(E.d.iter, E.d.disc, E.algo);
    E.sweep(0, -1, &pr);
    E.sweep(1, -1, &pr);
    CK(cudaStreamSynchronize(E.stream));
    E.iteration++;
    return pr;
}

double GpuEngine::exploitability(const HostSolver& host) {  // best_response.rs:255-287
    EngineImpl& E = *d_;
    const double denom = host.spot->pair_weight_sum();
    if (denom <= 0.0) return NAN;
    const bool raked = host.spot->config.tree.rake_pct > 0.0;
    double br[2], v[2] = {0, 0};
    for (int mode = 0; mode < (raked ? 2 : 1); mode++) {
        if (E.uncaptured) {
            E.record_eval(mode);
        } else {
            if (!E.g_eval[mode]) E.g_eval[mode] = E.capture(mode);
            CK(cudaGraphLaunch(E.g_eval[mode], E.stream));
        }
        E.reach_valid = false;
        CK(cudaStreamSynchronize(E.stream));
        E.check_err();
        for (int p = 0; p < 2; p++) (mode == 0 ? br[p] : v[p]) = E.h_dot[p] / denom;
    }
    if (raked) return ((br[0] - v[0]) + (br[1] - v[1])) / 2.0;
    return (br[0] + br[1]) / 2.0;
}

void GpuEngine::root_cfv(int p, int mode, float* out) {
    EngineImpl& E = *d_;
    E.sweep(p, mode, nullptr);
    E.reach_valid = false;
    CK(cudaMemcpyAsync(out, E.d.cfv, E.plan.nh[p] * sizeof(float), cudaMemcpyDeviceToHost, E.stream));
    CK(cudaStreamSynchronize(E.stream));
}

void GpuEngine::export_arena(int which, int p, float* out) {
    EngineImpl& E = *d_;
    fill_staging(which, p);
    E.d2h_large(out, E.staging, E.spot->tree.data_size[p] * 4);
}
// Device arena `which` of player p decoded into `staging` in the reference
// layout; nodes the engine does not hold (symmetric branches) are zero.
void GpuEngine::fill_staging(int which, int p) {
    EngineImpl& E = *d_;
    CK(cudaMemsetAsync(E.staging, 0, E.staging_len * 4, E.stream));
    const unsigned nb = (unsigned)E.plan.n_anodes[p];
    void* src = which == kRegrets ? E.ar.reg[p] : which == kStrategy ? E.ar.str[p] : E.ar.pred[p];
    if (nb && src) {
        if (E.fmt == kFmtF32) {
            k_to_host<float><<<nb, kThreads, 0, E.stream>>>((const float*)src, E.staging, E.xnodes[p], E.plan.nh[p]);
        } else if (E.fmt == kFmtFP8) {
            const float* sc = which == kRegrets ? E.ar.rscale[p] : which == kStrategy ? E.ar.sscale[p] : E.ar.pscale[p];
            k_decode_fp8_to_host<<<nb, kThreads, 0, E.stream>>>((const uint8_t*)src, sc, E.staging, E.xnodes[p],
                                                                 E.plan.nh[p]);
        } else if (which == kStrategy) {
            k_decode_to_host<uint16_t><<<nb, kThreads, 0, E.stream>>>((const uint16_t*)src, E.ar.sscale[p], E.staging,
                                                                       E.xnodes[p], E.plan.nh[p], 65535.0f);
        } else {
            const float* sc = which == kRegrets ? E.ar.rscale[p] : E.ar.pscale[p];
            k_decode_to_host<int16_t><<<nb, kThreads, 0, E.stream>>>((const int16_t*)src, sc, E.staging, E.xnodes[p],
                                                                      E.plan.nh[p], 32767.0f);
        }
        CK(cudaGetLastError());
    }
}

// ------------------------------------------------ node queries
// Average strategy of one action node (cfr.rs:679-726, the same rule the
// evaluation sweeps use) in the reference layout [action * nh + hand].
template <int FMT>
__global__ void k_node_avg_sigma(const void* str, float* out, int na, int nh) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nh) return;
    float sig[kSKA];
    s_average_sigma<FMT>(str, na, i, sig);
    for (int k = 0; k < na; k++) out[(size_t)k * nh + i] = sig[k];
}

void GpuEngine::node_average_strategy(uint32_t node, float* out) {
    EngineImpl& E = *d_;
    const Spot& sp = *E.spot;
    if (node >= sp.tree.size() || sp.tree.kind[node] != kAction) throw Error("not an action node");
    const int32_t s = E.plan.node_sidx[node];
    if (s < 0) throw Error("node " + std::to_string(node) + " has no device block (a symmetric branch)");
    const int p = sp.tree.player[node], na = sp.tree.nchild[node], nh = E.plan.nh[p];
    if (na > kSKA && E.fmt != kFmtF32 && E.fmt != kFmtI16) throw Error("node has more actions than the FP8 path takes");
    const XNode x = E.hx[p][(size_t)s];
    const unsigned grid = (unsigned)((nh + kThreads - 1) / kThreads);
    const size_t esz = (size_t)fmt_bytes(E.fmt);
    const void* blk = (const unsigned char*)E.ar.str[p] + x.dev_off * esz;
    if (na <= kSKA) {
        if (E.fmt == kFmtF32) k_node_avg_sigma<kDevF32><<<grid, kThreads, 0, E.stream>>>(blk, E.staging, na, nh);
        else if (E.fmt == kFmtFP8) k_node_avg_sigma<kDevFP8><<<grid, kThreads, 0, E.stream>>>(blk, E.staging, na, nh);
        else k_node_avg_sigma<kDevI16><<<grid, kThreads, 0, E.stream>>>(blk, E.staging, na, nh);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, E.staging, (size_t)na * nh * sizeof(float), cudaMemcpyDeviceToHost, E.stream));
        CK(cudaStreamSynchronize(E.stream));
        return;
    }
    // wide nodes (f32 / 16-bit arenas only): the block to the host, the same rule there
    std::vector<unsigned char> raw((size_t)na * nh * esz);
    CK(cudaMemcpyAsync(raw.data(), blk, raw.size(), cudaMemcpyDeviceToHost, E.stream));
    CK(cudaStreamSynchronize(E.stream));
    for (int i = 0; i < nh; i++) {
        if (E.fmt == kFmtF32) {
            const float* v = (const float*)raw.data() + (size_t)i * na;
            double sum = 0.0;
            for (int k = 0; k < na; k++) sum += (double)std::fmax(v[k], 0.0f);
            for (int k = 0; k < na; k++)
                out[(size_t)k * nh + i] = sum > 1e-12 ? (float)((double)std::fmax(v[k], 0.0f) / sum) : 1.0f / (float)na;
        } else {
            const uint16_t* q = (const uint16_t*)raw.data() + (size_t)i * na;
            unsigned sum = 0;
            for (int k = 0; k < na; k++) sum += q[k];
            const float inv = sum > 0 ? 1.0f / (float)sum : 0.0f;
            for (int k = 0; k < na; k++) out[(size_t)k * nh + i] = sum > 0 ? (float)q[k] * inv : 1.0f / (float)na;
        }
    }
}

void GpuEngine::node_sweep_values(uint32_t node, int p, int mode, float* cfv, float* reach0, float* reach1,
                                  float* child_cfv, uint8_t* child_ok) {
    EngineImpl& E = *d_;
    const Tree& t = E.spot->tree;
    if (node >= t.size() || E.plan.node_cslot[node] == kNoSlot && E.plan.node_rs[0][node] == kNoSlot)
        throw Error("node " + std::to_string(node) + " is not on the device (a symmetric branch or an in-place terminal)");
    if (mode != 0 && mode != 1) throw Error("invalid argument: sweep mode");
    E.levels_only = true;  // every node's slots (river programs keep river rounds in shared memory)
    try {
        E.sweep(p, mode, nullptr);  // down with the average strategies, up: best response (0) or average (1) for p
    } catch (...) {
        E.levels_only = false;
        throw;
    }
    E.levels_only = false;
    E.reach_valid = false;
    const int nh = E.plan.nh[p];
    const uint32_t cs = E.plan.node_cslot[node];
    if (cfv && cs != kNoSlot)
        CK(cudaMemcpyAsync(cfv, E.d.cfv + (size_t)cs * E.d.nh_max, nh * sizeof(float), cudaMemcpyDeviceToHost, E.stream));
    float* rr[2] = {reach0, reach1};
    for (int q = 0; q < 2; q++)
        if (rr[q])
            CK(cudaMemcpyAsync(rr[q], E.d.reach[q] + (size_t)E.plan.node_rs[q][node] * E.d.rstr[q],
                               E.plan.nh[q] * sizeof(float), cudaMemcpyDeviceToHost, E.stream));
    if (child_cfv && t.kind[node] == kAction && t.player[node] == p)
        for (int a = 0; a < t.nchild[node]; a++) {
            const uint32_t c = E.plan.node_cslot[t.child(node, a)];
            child_ok[a] = c != kNoSlot;
            if (c != kNoSlot)
                CK(cudaMemcpyAsync(child_cfv + (size_t)a * nh, E.d.cfv + (size_t)c * E.d.nh_max, nh * sizeof(float),
                                   cudaMemcpyDeviceToHost, E.stream));
        }
    CK(cudaStreamSynchronize(E.stream));
    E.check_err();
}

void GpuEngine::sweep_values(int p, int mode, const uint32_t* nodes, int n, float* out, uint8_t* ok) {
    EngineImpl& E = *d_;
    if (mode != 0 && mode != 1) throw Error("invalid argument: sweep mode");
    E.levels_only = true;
    try {
        E.sweep(p, mode, nullptr);
    } catch (...) {
        E.levels_only = false;
        throw;
    }
    E.levels_only = false;
    E.reach_valid = false;
    const int nh = E.plan.nh[p];
    for (int k = 0; k < n; k++) {
        const uint32_t c = nodes[k] < E.plan.node_cslot.size() ? E.plan.node_cslot[nodes[k]] : kNoSlot;
        ok[k] = c != kNoSlot;
        if (c != kNoSlot)
            CK(cudaMemcpyAsync(out + (size_t)k * nh, E.d.cfv + (size_t)c * E.d.nh_max, nh * sizeof(float),
                               cudaMemcpyDeviceToHost, E.stream));
    }
    CK(cudaStreamSynchronize(E.stream));
    E.check_err();
}

// ------------------------------------------------ .gto straight from / to HBM
// One block of a device save's image: dst <- src gathered through a hand
// permutation table, action by action (cfr.rs:806-871 copy_branch, with
// chains of copies composed down to a block in the image or one in the aux
// buffer: a lock, or a host block the engine does not hold).
struct SymOp {
    uint64_t dst, src;  // element offsets: dst in the image, src in the image or the aux buffer
    uint32_t na, tbl, aux, pad;
};
__global__ void k_sym_gather(float* img, const float* aux, const uint16_t* tbls, const SymOp* ops, int nh) {
    const SymOp op = ops[blockIdx.x];
    const uint16_t* T = tbls + (size_t)op.tbl * nh;
    const float* src = op.aux ? aux + op.src : img + op.src;
    const int n = (int)op.na * nh;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int a = e / nh, i = e - a * nh;
        img[op.dst + e] = src[(size_t)a * nh + T[i]];
    }
}

namespace {
// Device buffers and pinned host buffers owned for the length of one call.
struct TempDev {
    std::vector<void*> bufs;
    template <class T>
    T* put(const std::vector<T>& v, cudaStream_t st) {
        void* p = nullptr;
        CK(cudaMalloc(&p, std::max<size_t>(v.size(), 1) * sizeof(T)));
        bufs.push_back(p);
        if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        return (T*)p;
    }
    ~TempDev() {
        for (void* p : bufs) cudaFree(p);
    }
};
// Two pinned chunks and their events: the copy of one chunk overlaps the
// file I/O of the other.
struct PinnedPair {
    static constexpr size_t kChunk = size_t(8) << 20;  // floats (32 MiB)
    float* h[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    PinnedPair() {
        for (int b = 0; b < 2; b++) {
            CK(cudaMallocHost(&h[b], kChunk * sizeof(float)));
            CK(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
        }
    }
    ~PinnedPair() {
        for (int b = 0; b < 2; b++) {
            if (ev[b]) cudaEventDestroy(ev[b]);
            if (h[b]) cudaFreeHost(h[b]);
        }
    }
};
}  // namespace

void GpuEngine::save(const HostSolver& host, const std::string& path) {
    EngineImpl& E = *d_;
    if (E.plan.nshards > 1)
        throw Error("invalid argument: a shard holds part of the spot (sync each shard to the host solver, then save it)");
    if (E.leaf) throw Error("invalid argument: a depth-limited solve holds no subtrees below its turn leaves");
    CK(cudaStreamSynchronize(E.stream));
    E.check_err();
    const Spot& sp = *E.spot;
    const Tree& t = sp.tree;
    if (host.spot->tree.size() != t.size() || host.spot->tree.data_size[0] != t.data_size[0] ||
        host.spot->tree.data_size[1] != t.data_size[1])
        throw Error("invalid argument: the solver is not the one this GPU solver was built from");
    // The image of each arena, as the host path leaves it (sync_to_cpu, then
    // ensure_symmetric): the engine's blocks; with suit isomorphism, each
    // copy of ensure_symmetric in its order, composed with the copy that
    // produced its source until the source is a block of the image or a lock
    // (strategy sums); and the host's own values for the blocks neither
    // writes (children of a chance node for an already dealt card, which no
    // sweep visits).
    std::vector<std::vector<uint16_t>> tbl[2];
    std::map<std::vector<uint16_t>, uint32_t> tid[2];
    auto intern = [&](int p, std::vector<uint16_t>&& T) {
        auto it = tid[p].find(T);
        if (it != tid[p].end()) return it->second;
        const uint32_t k = (uint32_t)tbl[p].size();
        tid[p].emplace(T, k);
        tbl[p].push_back(std::move(T));
        return k;
    };
    for (int p = 0; p < 2; p++) {
        std::vector<uint16_t> id(E.plan.nh[p]);
        for (size_t i = 0; i < id.size(); i++) id[i] = (uint16_t)i;
        intern(p, std::move(id));
    }
    struct Src {
        uint32_t node, tbl;
        bool lock;
    };
    std::vector<SymOp> fill[2][2], copy[2][2];  // [regrets / strategy sums][player]
    std::vector<float> aux[2];                    // per arena kind: host blocks, then locks
    if (E.plan.iso_active) {
        std::unordered_map<uint32_t, Src> rsrc, ssrc;
        for (const auto& c : host.symmetric_copies()) {
            const int p = t.player[c.src];
            const auto& hk = sp.hand_perm[p][c.perm];
            auto compose = [&](uint32_t base) {
                const std::vector<uint16_t>& B = tbl[p][base];
                std::vector<uint16_t> T(hk.size());
                for (size_t i = 0; i < T.size(); i++) T[i] = B[hk[i]];
                return intern(p, std::move(T));
            };
            auto ri = rsrc.find(c.src);
            const Src r = ri != rsrc.end() ? ri->second : Src{c.src, 0, false};
            rsrc[c.dst] = {r.node, compose(r.tbl), false};
            if (host.locks.count(c.src)) {
                ssrc[c.dst] = {c.src, compose(0), true};
            } else {
                auto si = ssrc.find(c.src);
                const Src q = si != ssrc.end() ? si->second : Src{c.src, 0, false};
                ssrc[c.dst] = {q.node, compose(q.tbl), q.lock};
            }
        }
        for (uint32_t nd = 0; nd < t.size(); nd++) {
            if (t.kind[nd] != kAction || E.plan.node_sidx[nd] >= 0 || rsrc.count(nd)) continue;
            const int p = t.player[nd];
            const size_t cnt = (size_t)t.nchild[nd] * E.plan.nh[p];
            for (int w = 0; w < 2; w++) {
                const size_t at = aux[w].size();
                aux[w].resize(at + cnt);
                (w == 0 ? host.regrets[p] : host.strat[p]).read(nd, t.data_off[nd], cnt, aux[w].data() + at);
                fill[w][p].push_back({t.data_off[nd], at, t.nchild[nd], 0u, 1u, 0u});
            }
        }
        std::map<uint32_t, uint64_t> lock_at;
        for (int w = 0; w < 2; w++)
            for (const auto& kv : w == 0 ? rsrc : ssrc) {
                const uint32_t dst = kv.first;
                const Src& sr = kv.second;
                uint64_t src_off = t.data_off[sr.node];
                if (sr.lock) {
                    auto it = lock_at.find(sr.node);
                    if (it == lock_at.end()) {
                        const auto& lv = host.locks.at(sr.node);
                        it = lock_at.emplace(sr.node, (uint64_t)aux[1].size()).first;
                        aux[1].insert(aux[1].end(), lv.begin(), lv.end());
                    }
                    src_off = it->second;
                }
                copy[w][t.player[dst]].push_back({t.data_off[dst], src_off, t.nchild[dst], sr.tbl, sr.lock ? 1u : 0u, 0u});
            }
    }
    TempDev tmp;
    const uint16_t* dtbl[2] = {nullptr, nullptr};
    for (int p = 0; p < 2; p++) {
        std::vector<uint16_t> flat;
        for (const auto& T : tbl[p]) flat.insert(flat.end(), T.begin(), T.end());
        dtbl[p] = tmp.put(flat, E.stream);
    }
    const float* daux[2] = {tmp.put(aux[0], E.stream), tmp.put(aux[1], E.stream)};
    PinnedPair pin;
    host.save_stream(path, E.iteration, [&](int k, FILE* f) {
        const int p = k % 2, w = k < 2 ? 0 : 1;
        const uint64_t len = t.data_size[p];
        fill_staging(w == 0 ? kRegrets : kStrategy, p);
        for (const auto* ops : {&fill[w][p], &copy[w][p]})  // the copies read filled blocks: two launches
            if (!ops->empty()) {
                const SymOp* dops = tmp.put(*ops, E.stream);
                k_sym_gather<<<(unsigned)ops->size(), kThreads, 0, E.stream>>>(E.staging, daux[w], dtbl[p], dops,
                                                                              E.plan.nh[p]);
                CK(cudaGetLastError());
            }
        if (!write_arena_len(f, len)) return false;
        const size_t nc = (len + PinnedPair::kChunk - 1) / PinnedPair::kChunk;
        auto issue = [&](size_t j) {
            const size_t off = j * PinnedPair::kChunk, cnt = std::min<size_t>(PinnedPair::kChunk, len - off);
            CK(cudaMemcpyAsync(pin.h[j & 1], E.staging + off, cnt * 4, cudaMemcpyDeviceToHost, E.stream));
            CK(cudaEventRecord(pin.ev[j & 1], E.stream));
        };
        if (nc) issue(0);
        for (size_t j = 0; j < nc; j++) {
            if (j + 1 < nc) issue(j + 1);
            CK(cudaEventSynchronize(pin.ev[j & 1]));
            const size_t cnt = std::min<size_t>(PinnedPair::kChunk, len - j * PinnedPair::kChunk);
            if (fwrite(pin.h[j & 1], 4, cnt, f) != cnt) {
                CK(cudaStreamSynchronize(E.stream));
                return false;
            }
        }
        return true;
    });
    CK(cudaStreamSynchronize(E.stream));
}

void GpuEngine::load_arenas(std::istream& in, HostSolver& host) {
    EngineImpl& E = *d_;
    if (E.plan.nshards > 1) throw Error("invalid argument: a shard holds part of the spot (load on the host)");
    if (E.leaf) throw Error("invalid argument: a depth-limited solve holds no subtrees below its turn leaves");
    CK(cudaStreamSynchronize(E.stream));
    const Tree& t = E.spot->tree;
    // blocks the device does not hold, in arena order: they go to the host
    // arenas (a block split over two chunks is assembled first)
    struct Blk {
        uint64_t off;
        size_t cnt;
        uint32_t node;
    };
    std::vector<Blk> rest[2];
    for (uint32_t nd = 0; nd < t.size(); nd++)
        if (t.kind[nd] == kAction && E.plan.node_sidx[nd] < 0)
            rest[t.player[nd]].push_back({t.data_off[nd], (size_t)t.nchild[nd] * E.plan.nh[t.player[nd]], nd});
    for (auto& r : rest) std::sort(r.begin(), r.end(), [](const Blk& a, const Blk& b) { return a.off < b.off; });
    if (!rest[0].empty() || !rest[1].empty()) host.arenas_zero = false;
    PinnedPair pin;
    std::vector<float> part;
    for (int k = 0; k < 4; k++) {
        const int p = k % 2, which = k < 2 ? kRegrets : kStrategy;
        Arena& ha = which == kRegrets ? host.regrets[p] : host.strat[p];
        const uint64_t len = read_arena_len(in, t.data_size[p]);
        const size_t nc = (len + PinnedPair::kChunk - 1) / PinnedPair::kChunk;
        size_t b = 0;  // next block of rest[p]
        for (size_t j = 0; j < nc; j++) {
            const size_t off = j * PinnedPair::kChunk, cnt = std::min<size_t>(PinnedPair::kChunk, len - off);
            float* hb = pin.h[j & 1];
            if (j >= 2) CK(cudaEventSynchronize(pin.ev[j & 1]));  // its previous copy has left the buffer
            if (!in.read((char*)hb, (std::streamsize)(cnt * 4))) throw Error("truncated arena");
            CK(cudaMemcpyAsync(E.staging + off, hb, cnt * 4, cudaMemcpyHostToDevice, E.stream));
            CK(cudaEventRecord(pin.ev[j & 1], E.stream));
            for (; b < rest[p].size() && rest[p][b].off < off + cnt; b++) {
                const Blk& x = rest[p][b];
                if (x.off >= off && x.off + x.cnt <= off + cnt) {
                    ha.write(x.node, x.off, x.cnt, hb + (x.off - off));
                    continue;
                }
                // split block: its parts in this chunk and the next ones
                const uint64_t lo = std::max<uint64_t>(x.off, off), hi = std::min<uint64_t>(x.off + x.cnt, off + cnt);
                if (x.off >= off) part.assign(x.cnt, 0.0f);
                std::memcpy(part.data() + (lo - x.off), hb + (lo - off), (hi - lo) * sizeof(float));
                if (x.off + x.cnt > off + cnt) break;  // continues in the next chunk
                ha.write(x.node, x.off, x.cnt, part.data());
            }
        }
        E.encode_staging(which, p);
        CK(cudaStreamSynchronize(E.stream));
    }
    for (int p = 0; p < 2; p++)  // the file holds no predictions: PCFR+ restarts them at zero
        if (E.ar.pred[p]) {
            CK(cudaMemsetAsync(E.ar.pred[p], 0, E.plan.arena_len[p] * (size_t)fmt_bytes(E.fmt), E.stream));
            if (E.ar.pscale[p]) CK(cudaMemsetAsync(E.ar.pscale[p], 0, std::max<uint64_t>(E.plan.n_anodes[p], 1) * 4, E.stream));
        }
    E.reach_valid = false;
    CK(cudaStreamSynchronize(E.stream));
    E.check_err();
}

// ------------------------------------------------ allocation-free node read
// Scratch of read_node_static: one action node's block decoded to f32 in the
// reference layout [action * nh + hand].  File-scope device memory, so a call
// allocates nothing; every element that is copied out is written by the same
// call first, so nothing in it has to start at zero.  One array per device,
// shared by every engine on that device: calls that overlap in time race.
static __device__ __align__(256) float g_node_scratch[kNodeScratchElems];

// Variant of k_to_host / k_decode_to_host for one node, writing into the
// scratch at offset 0 (scale == nullptr: an f32 arena, copied as is).
template <class T>
__global__ void k_node_to_scratch(const T* dev, const float* scale, float div, float* dst, XNode x, int nh) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nh) return;
    const float kq = scale ? scale[x.sidx] / div : 1.0f;
    for (uint32_t k = 0; k < x.na; k++) {
        const T v = dev[x.dev_off + (size_t)i * x.na + k];
        dst[(size_t)k * nh + i] = scale ? (float)v * kq : (float)v;
    }
}
// FP8 arenas: e4m3 value * (scale / 448), as k_decode_fp8_to_host.
__global__ void k_node_fp8_to_scratch(const uint8_t* dev, const float* scale, float* dst, XNode x, int nh) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nh) return;
    const float kq = scale[x.sidx] / 448.0f;
    for (uint32_t k = 0; k < x.na; k++) dst[(size_t)k * nh + i] = e4m3_to_f32(dev[x.dev_off + (size_t)i * x.na + k]) * kq;
}
constexpr int kMaxDevices = 64;

// Per-device address of g_node_scratch, resolved once with that device current.
static float* node_scratch_ptr(int device) {
    static std::mutex mu;
    static float* ptrs[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices) throw Error("device ordinal out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (!ptrs[device]) {
        void* p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_node_scratch);
        if (rc != cudaSuccess) throw Error(std::string("cuda: cudaGetSymbolAddress(node scratch): ") + cudaGetErrorString(rc));
        ptrs[device] = (float*)p;
    }
    return ptrs[device];
}

size_t GpuEngine::read_node_static(int which, uint32_t node, float* out, size_t out_len) {
    EngineImpl& E = *d_;
    const Spot& sp = *E.spot;
    if (node >= sp.tree.size() || sp.tree.kind[node] != kAction) throw Error("node " + std::to_string(node) + " is not an action node");
    const int p = sp.tree.player[node];
    const int32_t s = E.plan.node_sidx[node];
    if (s < 0)
        throw Error("node " + std::to_string(node) +
                    " has no block on this engine's device (a symmetric branch the engine skips, or a node of "
                    "another shard)");
    if (which == kPreds && !E.pcfr) throw Error("the engine keeps no predictions (not PCFR+)");
    const XNode x = E.hx[p][(size_t)s];
    const int nh = E.plan.nh[p];
    const size_t n = (size_t)x.na * (size_t)nh;
    if (n > kNodeScratchElems)
        throw Error("node " + std::to_string(node) + " block has " + std::to_string(n) + " elements, more than the " +
                    std::to_string(kNodeScratchElems) + "-element static scratch");
    if (out_len < n) throw Error("invalid argument: output holds " + std::to_string(out_len) + " floats, node needs " +
                                 std::to_string(n));
    int dev = -1;
    CK(cudaGetDevice(&dev));
    cudaPointerAttributes attr;
    CK(cudaPointerGetAttributes(&attr, E.d.cfv));
    if (attr.device != dev) throw Error("invalid argument: the engine's device is not the current device");
    float* scratch = node_scratch_ptr(dev);
    const void* src = which == kRegrets ? E.ar.reg[p] : which == kStrategy ? E.ar.str[p] : E.ar.pred[p];
    const unsigned grid = (unsigned)((nh + kThreads - 1) / kThreads);
    if (E.fmt == kFmtF32) {
        k_node_to_scratch<float><<<grid, kThreads, 0, E.stream>>>((const float*)src, nullptr, 1.0f, scratch, x, nh);
    } else if (E.fmt == kFmtFP8) {
        const float* sc = which == kRegrets ? E.ar.rscale[p] : which == kStrategy ? E.ar.sscale[p] : E.ar.pscale[p];
        k_node_fp8_to_scratch<<<grid, kThreads, 0, E.stream>>>((const uint8_t*)src, sc, scratch, x, nh);
    } else {
        const float* sc = which == kRegrets ? E.ar.rscale[p] : which == kStrategy ? E.ar.sscale[p] : E.ar.pscale[p];
        if (which == kStrategy)
            k_node_to_scratch<uint16_t><<<grid, kThreads, 0, E.stream>>>((const uint16_t*)src, sc, 65535.0f, scratch, x, nh);
        else
            k_node_to_scratch<int16_t><<<grid, kThreads, 0, E.stream>>>((const int16_t*)src, sc, 32767.0f, scratch, x, nh);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, scratch, n * sizeof(float), cudaMemcpyDeviceToHost, E.stream));
    CK(cudaStreamSynchronize(E.stream));
    E.check_err();  // a sticky device error of an earlier iteration is reported, not returned as data
    return n;
}

void GpuEngine::sync_to_cpu(HostSolver& host, bool strategy_only) {  // gpu/mod.rs:845-886
    EngineImpl& E = *d_;
    CK(cudaStreamSynchronize(E.stream));
    E.check_err();
    const Spot& sp = *E.spot;
    const Tree& t = sp.tree;
    for (int p = 0; p < 2; p++) {
        const int nh = E.plan.nh[p];
        for (int which = strategy_only ? 1 : 0; which < (E.pcfr && !strategy_only ? 3 : 2); which++) {
            Arena& ha = which == kRegrets ? host.regrets[p] : which == kStrategy ? host.strat[p]
                                                             : (host.ensure_preds(), host.preds[p]);
            const unsigned nb = (unsigned)E.plan.n_anodes[p];
            if (!nb) continue;
            void* src = which == kRegrets ? E.ar.reg[p] : which == kStrategy ? E.ar.str[p] : E.ar.pred[p];
            // Without suit isomorphism or shards every action node is on the
            // device, so the reference-layout image is the whole host arena and
            // lands there directly; otherwise it goes through a temporary and
            // only the device's nodes are copied (the symmetric branches and
            // the other shards' nodes keep theirs).
            const bool whole = !E.plan.iso_active && E.plan.nshards == 1;
            if (E.fmt == kFmtI16 && ha.kind != 0) {
                // 16-bit on both sides: quants and scales move exactly
                k_to_host<uint16_t><<<nb, kThreads, 0, E.stream>>>((const uint16_t*)src, (uint16_t*)E.staging, E.xnodes[p], nh);
                std::vector<float> sc(E.plan.n_anodes[p]);
                const float* dsc = which == kRegrets ? E.ar.rscale[p] : which == kStrategy ? E.ar.sscale[p] : E.ar.pscale[p];
                CK(cudaMemcpyAsync(sc.data(), dsc, sc.size() * 4, cudaMemcpyDeviceToHost, E.stream));
                uint16_t* harena = ha.kind == 1 ? (uint16_t*)ha.qi.data() : ha.qu.data();
                std::vector<uint16_t> tmp(whole ? 0 : t.data_size[p]);
                CK(cudaStreamSynchronize(E.stream));
                E.d2h_large(whole ? harena : tmp.data(), E.staging, t.data_size[p] * 2);
                for (uint64_t s = 0; s < E.plan.n_anodes[p]; s++) {
                    const uint32_t nd = E.plan.anode_id[p][s];
                    if (!whole) {
                        const size_t off = t.data_off[nd], cnt = (size_t)t.nchild[nd] * nh;
                        std::memcpy(harena + off, tmp.data() + off, cnt * 2);
                    }
                    ha.scale[nd] = sc[s];
                }
                continue;
            }
            if (whole && ha.kind == 0) {
                export_arena(which, p, ha.f.data());
                continue;
            }
            std::vector<float> img(t.data_size[p]);
            export_arena(which, p, img.data());
            for (uint64_t s = 0; s < E.plan.n_anodes[p]; s++) {
                const uint32_t nd = E.plan.anode_id[p][s];
                ha.write(nd, t.data_off[nd], (size_t)t.nchild[nd] * nh, img.data() + t.data_off[nd]);
            }
        }
    }
    host.iteration = E.iteration;
    host.arenas_zero = false;
    if (E.plan.iso_active) host.sym_dirty = true;
}

void GpuEngine::synchronize() {
    CK(cudaStreamSynchronize(d_->stream));
    d_->check_err();
}
void GpuEngine::update_locks(const HostSolver& host) { d_->upload_locks(host); }
uint32_t GpuEngine::iteration() const { return d_->iteration; }
int GpuEngine::format() const { return d_->fmt == kFmtI16 && d_->ar.sr ? kFmtI16SR : d_->fmt; }
bool GpuEngine::fused() const { return d_->plan.fused; }
const Plan& GpuEngine::plan() const { return d_->plan; }
const Spot* GpuEngine::plan_spot() const { return d_->spot; }
uint64_t GpuEngine::device_bytes() const { return d_->bytes; }
void GpuEngine::discounts(float* out3) {
    CK(cudaMemcpyAsync(out3, d_->d.disc, 3 * sizeof(float), cudaMemcpyDeviceToHost, d_->stream));
    CK(cudaStreamSynchronize(d_->stream));
}
double GpuEngine::iter_bytes() const {
    // Algorithmic bytes of one iteration: sigma reads of both arenas in both
    // down sweeps, read+write of the traverser's regrets and sums, one
    // opponent-reach read and one cfv write per terminal per traversal.
    const Plan& P = d_->plan;
    const double b = (double)fmt_bytes(d_->fmt);
    const double D = (double)(P.visited_action_elems[0] + P.visited_action_elems[1]);
    double bytes = 2.0 * D * b + 2.0 * D * (b + b) + 2.0 * (double)P.visited_terminals * (P.nh[0] + P.nh[1]) * 4.0;
    if (d_->fmt != kFmtF32) bytes += 8.0 * (double)(P.n_anodes[0] + P.n_anodes[1]) * 2.0;
    return bytes;
}

uint64_t estimate_vram(const Spot& spot) {  // same role as game.rs:365-373, for this engine's layout
    Plan P = build_plan(spot, true, kFuseFolds);  // the default (staged) engine's plan
    uint64_t b = P.n_cslots * (uint64_t)P.nh_max * 4 + P.n_rslots[0] * (uint64_t)P.nh[0] * 4 +
                 P.n_rslots[1] * (uint64_t)P.nh[1] * 4;
    b += (P.arena_len[0] + P.arena_len[1]) * 2 * 4;
    return b + 512ull * 1024 * 1024;
}
bool vram_info_mb(uint64_t* free_mb, uint64_t* total_mb) {
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) return false;
    *free_mb = f / 1000000;
    *total_mb = t / 1000000;
    return true;
}


// ---------------------------------------------------------------------------
// Batched engine (cfr_batch.cuh): many engines' CFR iterations in one
// persistent kernel launch per iteration.

struct BatchImpl {
    std::vector<GpuEngine*> eng;
    std::vector<EngineImpl*> E;
    int fmt = -1;
    BatchShape shape;
    cudaStream_t stream = nullptr;
    std::vector<void*> owned;  // device buffers of the current set
    size_t bytes = 0;
    BSpot* spots = nullptr;
    BSeg* segs = nullptr;
    unsigned* ctl = nullptr;
    size_t nctl = 0;
    int nseg = 0;
    unsigned nticket = 0;
    uint64_t nrecord = 0;
    size_t smem = 0;
    int grid = 0;
    cudaGraphExec_t graph = nullptr;
    unsigned h_ctl[4] = {0, 0, 0, 0};
    ~BatchImpl() {
        release();
        if (stream) cudaStreamDestroy(stream);
    }
    void release() {
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        for (void* p : owned) cudaFree(p);
        owned.clear();
        spots = nullptr;
        segs = nullptr;
        ctl = nullptr;
        nseg = 0;
        nticket = 0;
        nrecord = 0;
    }
    template <int FMT>
    static const void* kernel() { return (const void*)kb_iterate<FMT>; }
    const void* kernel_fn() const {
        return fmt == kFmtF32 ? kernel<kDevF32>() : fmt == kFmtFP8 ? kernel<kDevFP8>() : kernel<kDevI16>();
    }
    int occupancy() const {
        int n = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel_fn(), kBThreads, smem));
        return n;
    }
    void build() {
        release();
        if (eng.empty()) return;
        if (!stream) CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        std::vector<BSpot> hs(E.size());
        smem = 16;
        std::vector<const Plan*> plans;
        for (size_t s = 0; s < E.size(); s++) {
            const EngineImpl& X = *E[s];
            BSpot& b = hs[s];
            std::memset(&b, 0, sizeof(b));
            b.d = X.d;
            b.ar = X.ar;
            b.snodes = X.snodes;
            b.edge = X.edge;
            b.show = X.show;
            b.show_batch = X.show_batch;
            b.chance = X.chance;
            b.msort = (int)X.plan.max_sorted;
            b.algo = X.algo;
            smem = std::max({smem, X.st_mine_smem, X.st_opp_smem, X.st_down_smem, X.show_pair_smem, X.chance_smem});
            plans.push_back(&X.plan);
        }
        // segments ordered by step, then spot; a segment's tickets wait for
        // the spot's tickets of its earlier steps (host/plan.cpp)
        std::vector<BatchSegment> q;
        const uint64_t t = batch_queue(plans, shape.tile, q, &nrecord);
        std::vector<BSeg> hg(q.size());
        for (size_t k = 0; k < q.size(); k++) {
            BSeg& g = hg[k];
            std::memset(&g, 0, sizeof(g));
            g.first = (uint32_t)q[k].first;
            g.start = q[k].start;
            g.count = q[k].count;
            g.need = q[k].need;
            g.spot = (uint16_t)q[k].spot;
            g.kind = (uint8_t)q[k].kind;
            g.p = (uint8_t)q[k].p;
            g.tile = (uint16_t)q[k].tile;
        }
        if (t >= 0xFFFFFFFFull) throw Error("batch: too many tickets in one iteration");
        nticket = (unsigned)t;
        nseg = (int)hg.size();
        spots = dupload(hs, owned, &bytes);
        segs = dupload(hg, owned, &bytes);
        nctl = (size_t)kBCtlDone + E.size();
        ctl = (unsigned*)dalloc(nctl * sizeof(unsigned), owned, &bytes);
        set_smem(kernel_fn(), smem);
        int dev = 0, nsm = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const int occ = occupancy();
        if (occ < 1) throw Error("batch: the kernel does not fit an SM (" + std::to_string(smem) + " B shared memory)");
        const int per = shape.ctas_per_sm > 0 ? std::min(shape.ctas_per_sm, occ) : occ;
        grid = nsm * per;
        // the iteration's graph: control words zeroed, then the kernel
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaMemsetAsync(ctl, 0, nctl * sizeof(unsigned), stream);
        if (fmt == kFmtF32)
            kb_iterate<kDevF32><<<grid, kBThreads, smem, stream>>>(spots, segs, nseg, nticket, ctl);
        else if (fmt == kFmtFP8)
            kb_iterate<kDevFP8><<<grid, kBThreads, smem, stream>>>(spots, segs, nseg, nticket, ctl);
        else
            kb_iterate<kDevI16><<<grid, kBThreads, smem, stream>>>(spots, segs, nseg, nticket, ctl);
        const cudaError_t le = cudaGetLastError();
        CK(cudaStreamEndCapture(stream, &g));
        if (le != cudaSuccess) {
            cudaGraphDestroy(g);
            throw Error(std::string("cuda: ") + cudaGetErrorString(le) + " launching the batch kernel");
        }
        const cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        CK(ie);
    }
    // Every engine's own work done and its reach current (after an
    // evaluation sweep an engine primes its reach first, as iterate does).
    void ready() {
        const cudaError_t pend = cudaGetLastError();
        if (pend != cudaSuccess)
            throw Error(std::string("cuda: ") + cudaGetErrorString(pend) + " (pending before the batched launch)");
        for (EngineImpl* X : E) {
            X->prime();
            CK(cudaStreamSynchronize(X->stream));
        }
    }
    void finish(int n) {
        CK(cudaMemcpyAsync(h_ctl, ctl, sizeof(h_ctl), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        for (EngineImpl* X : E) X->iteration += (uint32_t)n;
        if (h_ctl[kBCtlAbort]) {
            for (EngineImpl* X : E) X->check_err();  // a copy's error, with its message
            throw Error((h_ctl[kBCtlErr] & 4u) ? "timeout: a batched step waited too long for its spot's earlier steps"
                                               : "timeout: the batched iteration stopped");
        }
    }
};

BatchKernel::BatchKernel() : d_(new BatchImpl()) {}
BatchKernel::~BatchKernel() = default;

std::string BatchKernel::unsupported(const GpuEngine& e) {
    const EngineImpl& X = *e.d_;
    if (!X.staged) return "the spot's engine is not the staged engine (nodes of more than 4 actions, or another kind)";
    if (X.river) return "river programs are not batched";
    if (X.leaf) return "depth-limited engines are not batched";
    if (X.reducer) return "sharded engines are not batched";
    if (!X.term64) return "f32 terminal sums are not batched";
    for (const Span& s : X.plan.fold_span)
        if (s.count) return "fold terminals with slots of their own are not batched";
    return "";
}
void BatchKernel::configure(const std::vector<GpuEngine*>& engines, const BatchShape& shape) {
    BatchImpl& B = *d_;
    B.shape = shape;
    if (engines.size() > 65535) throw Error("invalid argument: at most 65535 spots in one batch");
    int fmt = -1;
    for (GpuEngine* e : engines) {
        if (!e) throw Error("invalid argument: null engine");
        const std::string why = unsupported(*e);
        if (!why.empty()) throw Error("invalid argument: " + why);
        if (fmt >= 0 && e->d_->fmt != fmt) throw Error("invalid argument: the batch's engines differ in arena format");
        fmt = e->d_->fmt;
    }
    B.eng = engines;
    B.E.clear();
    for (GpuEngine* e : engines) B.E.push_back(e->d_.get());
    if (fmt >= 0) B.fmt = fmt;
    B.build();
}
void BatchKernel::configure_shape(const BatchShape& s) {
    d_->shape = s;
    d_->build();
}
BatchShape BatchKernel::shape() const { return d_->shape; }
int BatchKernel::max_ctas_per_sm() const { return d_->eng.empty() ? 0 : d_->occupancy(); }
int BatchKernel::grid() const { return d_->grid; }
size_t BatchKernel::tickets() const { return d_->nticket; }
uint64_t BatchKernel::records() const { return d_->nrecord; }
void BatchKernel::iterate(int n) {
    BatchImpl& B = *d_;
    if (B.eng.empty() || n <= 0) return;
    B.ready();
    for (int k = 0; k < n; k++) CK(cudaGraphLaunch(B.graph, B.stream));
    B.finish(n);
}
double BatchKernel::time_iterations(int n) {
    BatchImpl& B = *d_;
    if (B.eng.empty() || n <= 0) return 0.0;
    B.ready();
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, B.stream));
    for (int k = 0; k < n; k++) CK(cudaGraphLaunch(B.graph, B.stream));
    CK(cudaEventRecord(b, B.stream));
    CK(cudaEventSynchronize(b));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    B.finish(n);
    return ms;
}

}  // namespace gtob
