// C ABI (include/gtob.h): thin wrappers turning C++ exceptions into status
// codes plus a thread-local message, the way the reference's Result<_, String>
// errors reach its callers.
#include "../../../include/gtob.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <thread>
#include <fstream>
#include <memory>
#include <string>

#include "../kernels/engine.hpp"
#include "../kernels/leafnet.hpp"
#include "batch.hpp"
#include "core.hpp"
#include "query.hpp"
#include "shard.hpp"
#include "solver.hpp"

using namespace gtob;

struct gtob_spot { std::shared_ptr<Spot> s; };
struct gtob_solver { std::unique_ptr<HostSolver> v; };
struct gtob_gpu { std::unique_ptr<GpuEngine> e; };
struct gtob_net {
    std::shared_ptr<LeafNet> n;
};
struct gtob_shards {
    std::vector<std::unique_ptr<GpuEngine>> e;
    int device = 0;
    // runs f(shard) for every shard on its own thread (the host exchange
    // needs them all at once); the first error is rethrown
    template <class F>
    void all(F f) {
        std::vector<std::exception_ptr> errs(e.size());
        std::vector<std::thread> ts;
        for (size_t k = 0; k < e.size(); k++)
            ts.emplace_back([&, k] {
                try {
                    const cudaError_t rc = cudaSetDevice(device);
                    if (rc != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(rc));
                    f((int)k);
                } catch (...) {
                    errs[k] = std::current_exception();
                }
            });
        for (auto& t : ts) t.join();
        for (auto& x : errs)
            if (x) std::rethrow_exception(x);
    }
};


static thread_local std::string g_err;

template <class T>
static void put(T* dst, const std::vector<T>& v) {
    if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(T));
}

static int classify(const std::string& m) {
    if (m.rfind("timeout:", 0) == 0) return GTOB_ETIMEOUT_QUEUE;
    if (m.rfind("cuda: out of memory", 0) == 0 || m.find("out of memory") != std::string::npos) return GTOB_ENOMEM_DEVICE;
    if (m.rfind("cuda:", 0) == 0) return GTOB_ECUDA;
    if (m.rfind("io:", 0) == 0 || m.find("cannot open") != std::string::npos || m.find("write failed") != std::string::npos ||
        m.find("rename failed") != std::string::npos || m.find("cannot create") != std::string::npos)
        return GTOB_EIO;
    return GTOB_EINVAL;
}
#define API_BEGIN try {
#define API_END                              \
    }                                        \
    catch (const std::exception& ex) {       \
        g_err = ex.what();                   \
        return classify(g_err);              \
    }                                        \
    catch (...) {                            \
        g_err = "unknown error";             \
        return GTOB_EINVAL;                  \
    }                                        \
    return GTOB_OK;
#define REQUIRE(c)                                               \
    if (!(c)) {                                                  \
        g_err = "invalid argument: " #c;                         \
        return GTOB_EINVAL;                                      \
    }

extern "C" {

const char* gtob_last_error(void) { return g_err.c_str(); }
const char* gtob_kernel_name(int k) { return (k >= 0 && k < 7) ? kKernelNames[k] : ""; }
const char* gtob_version(void) { return "gtob 0.1 sm_100a"; }

int gtob_spot_from_json(const char* js, uint64_t max_nodes, int lenient, gtob_spot** out) {
    REQUIRE(js && out);
    *out = nullptr;
    API_BEGIN
    SpotConfig cfg = config_from_json(json::parse(js));
    auto s = build_spot(cfg, max_nodes, lenient != 0);
    *out = new gtob_spot{std::shared_ptr<Spot>(s.release())};
    API_END
}
void gtob_spot_free(gtob_spot* s) { delete s; }
int gtob_spot_info_get(const gtob_spot* s, gtob_spot_info* o) {
    REQUIRE(s && o);
    const Spot& sp = *s->s;
    o->num_nodes = sp.tree.size();
    o->num_action_nodes = sp.num_action_nodes();
    o->num_children = sp.tree.children.size();
    o->num_actions = sp.tree.act_kind.size();
    o->data_size[0] = sp.tree.data_size[0];
    o->data_size[1] = sp.tree.data_size[1];
    o->num_hands[0] = (uint32_t)sp.hands[0].size();
    o->num_hands[1] = (uint32_t)sp.hands[1].size();
    o->root_street = (uint32_t)sp.tree.root_street;
    o->num_suit_perms = (uint32_t)sp.perms.size();
    return GTOB_OK;
}
int gtob_spot_tree(const gtob_spot* s, uint8_t* kind, uint8_t* player, uint8_t* street, uint8_t* nchild,
                   uint32_t* cs, uint32_t* as, uint64_t* doff, double* p0, double* p1, double* tw, double* tl,
                   double* tt) {
    REQUIRE(s);
    const Tree& t = s->s->tree;
    put(kind, t.kind); put(player, t.player); put(street, t.street); put(nchild, t.nchild);
    put(cs, t.child_start); put(as, t.action_start); put(doff, t.data_off);
    put(p0, t.put0); put(p1, t.put1); put(tw, t.twin); put(tl, t.tlose); put(tt, t.ttie);
    return GTOB_OK;
}
int gtob_spot_children(const gtob_spot* s, uint32_t* out) {
    REQUIRE(s && out);
    put(out, s->s->tree.children);
    return GTOB_OK;
}
int gtob_spot_actions(const gtob_spot* s, int32_t* kind, double* amount) {
    REQUIRE(s);
    const Tree& t = s->s->tree;
    for (size_t i = 0; i < t.act_kind.size(); i++) {
        if (kind) kind[i] = t.act_kind[i];
        if (amount) amount[i] = t.act_amount[i];
    }
    return GTOB_OK;
}
int gtob_spot_hands(const gtob_spot* s, int p, uint8_t* c1, uint8_t* c2, float* w, uint32_t* same) {
    REQUIRE(s && (p == 0 || p == 1));
    const Hands& h = s->s->hands[p];
    put(c1, h.c1); put(c2, h.c2); put(w, h.w); put(same, s->s->same[p]);
    return GTOB_OK;
}
int gtob_spot_suit_perms(const gtob_spot* s, uint8_t* perms4, uint16_t* hp0, uint16_t* hp1) {
    REQUIRE(s);
    const Spot& sp = *s->s;
    for (size_t k = 0; k < sp.perms.size(); k++) {
        if (perms4) std::memcpy(perms4 + 4 * k, sp.perms[k].data(), 4);
        if (hp0) std::memcpy(hp0 + k * sp.hands[0].size(), sp.hand_perm[0][k].data(), 2 * sp.hands[0].size());
        if (hp1) std::memcpy(hp1 + k * sp.hands[1].size(), sp.hand_perm[1][k].data(), 2 * sp.hands[1].size());
    }
    return GTOB_OK;
}
int gtob_spot_river(const gtob_spot* s, int p, const uint8_t* dealt, int nd, uint32_t* str, uint16_t* idx) {
    REQUIRE(s && (p == 0 || p == 1) && nd >= 0 && nd <= 2);
    API_BEGIN
    const RiverBoard& rb = s->s->river_at(dealt, nd);
    put(str, rb.str[p]);
    put(idx, rb.idx[p]);
    return (int)rb.str[p].size();
    API_END
}
double gtob_spot_pair_weight_sum(const gtob_spot* s) { return s ? s->s->pair_weight_sum() : 0.0; }
uint32_t gtob_evaluate7(const uint8_t* c) { return eval7(c); }
int gtob_parse_range(const char* text, float* w) {
    REQUIRE(text && w);
    API_BEGIN
    auto v = parse_range_weights(text);
    std::memcpy(w, v.data(), sizeof(float) * 1326);
    API_END
}
uint64_t gtob_estimate_vram(const gtob_spot* s) {
    if (!s) return 0;
    try {
        return estimate_vram(*s->s);
    } catch (...) {
        return 0;
    }
}
int gtob_vram_info_mb(uint64_t* f, uint64_t* t) {
    REQUIRE(f && t);
    if (!vram_info_mb(f, t)) {
        g_err = "cuda: no device";
        return GTOB_ECUDA;
    }
    return GTOB_OK;
}

int gtob_solver_new(gtob_spot* s, int storage, int algo, int use_iso, gtob_solver** out) {
    REQUIRE(s && out && (storage == 0 || storage == 1) && algo >= 0 && algo <= 2);
    *out = nullptr;
    API_BEGIN
    *out = new gtob_solver{std::make_unique<HostSolver>(s->s, storage, algo, use_iso != 0)};
    API_END
}
void gtob_solver_free(gtob_solver* v) { delete v; }
uint32_t gtob_solver_iteration(const gtob_solver* v) { return v ? v->v->iteration : 0; }
int gtob_solver_set_iteration(gtob_solver* v, uint32_t it) {
    REQUIRE(v);
    v->v->iteration = it;
    return GTOB_OK;
}
uint64_t gtob_solver_arena_bytes(const gtob_solver* v) { return v ? v->v->arena_bytes() : 0; }
int gtob_solver_get_arena(const gtob_solver* v, int which, int p, float* out) {
    REQUIRE(v && out && which >= 0 && which <= 2 && (p == 0 || p == 1));
    API_BEGIN
    v->v->arena_f32(which, p, out);
    API_END
}
int gtob_solver_set_arena(gtob_solver* v, int which, int p, const float* in) {
    REQUIRE(v && in && which >= 0 && which <= 2 && (p == 0 || p == 1));
    API_BEGIN
    v->v->set_arena_f32(which, p, in);
    API_END
}
static int check_action_node(const gtob_solver* v, uint32_t node) {
    const Tree& t = v->v->spot->tree;
    if (node >= t.size() || t.kind[node] != kAction) {
        g_err = "node " + std::to_string(node) + " is not an action node";
        return GTOB_EINVAL;
    }
    return GTOB_OK;
}
int gtob_solver_average_strategy(const gtob_solver* v, uint32_t node, float* out) {
    REQUIRE(v && out);
    if (int r = check_action_node(v, node)) return r;
    v->v->average_strategy(node, out);
    return GTOB_OK;
}
int gtob_solver_solved_strategy(const gtob_solver* v, uint32_t node, float* out) {
    REQUIRE(v && out);
    if (int r = check_action_node(v, node)) return r;
    v->v->solved_strategy(node, out);
    return GTOB_OK;
}
int gtob_solver_lock_node(gtob_solver* v, const int32_t* steps, int ns, int mode, const float* freqs, int nf,
                          const char* edits_json, const char* label, uint32_t* node_out) {
    REQUIRE(v && ns >= 0 && (ns == 0 || steps) && mode >= 0 && mode <= 2 && (nf == 0 || freqs));
    API_BEGIN
    std::vector<int> st(steps, steps + ns);
    std::vector<float> fr(freqs, freqs + nf);
    std::vector<std::pair<std::string, std::vector<float>>> edits;
    if (mode == 2) {
        if (!edits_json) throw Error("hand edits required");
        json::Value e = json::parse(edits_json);
        for (auto& x : e.arr) {
            if (x.kind != json::Value::ARR || x.arr.size() != 2 || x.arr[0].kind != json::Value::STR)
                throw Error("edit must be [combo, [freqs...]]");
            std::vector<float> f;
            for (auto& y : x.arr[1].arr) f.push_back((float)y.num);
            edits.push_back({x.arr[0].str, f});
        }
    }
    uint32_t n = v->v->lock_node(st, mode, fr, edits, label ? label : "");
    if (node_out) *node_out = n;
    API_END
}
int gtob_solver_set_lock(gtob_solver* v, uint32_t node, const float* sigma, uint64_t n, const char* label) {
    REQUIRE(v && sigma);
    API_BEGIN
    std::vector<std::pair<uint32_t, std::vector<float>>> l{{node, std::vector<float>(sigma, sigma + n)}};
    validate_locks(*v->v->spot, l);
    v->v->locks[node] = l[0].second;
    v->v->lock_labels[node] = label ? label : "";
    v->v->sym_dirty = true;
    API_END
}
int gtob_solver_clear_locks(gtob_solver* v) {
    REQUIRE(v);
    if (!v->v->locks.empty()) v->v->sym_dirty = true;
    v->v->locks.clear();
    v->v->lock_labels.clear();
    return GTOB_OK;
}
int gtob_solver_num_locks(const gtob_solver* v) { return v ? (int)v->v->locks.size() : 0; }
int gtob_solver_ensure_symmetric(gtob_solver* v) {
    REQUIRE(v);
    API_BEGIN
    v->v->ensure_symmetric();
    API_END
}
int gtob_save(const gtob_solver* v, const char* path) {
    REQUIRE(v && path);
    API_BEGIN
    v->v->save(path);
    API_END
}
int gtob_load(const char* path, int storage, gtob_solver** out) {
    REQUIRE(path && out && (storage == 0 || storage == 1));
    *out = nullptr;
    API_BEGIN
    *out = new gtob_solver{HostSolver::load(path, storage)};
    API_END
}

int gtob_gpu_node_values(gtob_gpu* g, const gtob_solver* v, const int* steps, int nsteps, gtob_node_info* info,
                         float* reach0, float* reach1, float* valid0, float* valid1, float* eq0, float* eq1,
                         float* ev0, float* ev1, float* strategy, float* action_ev) {
    REQUIRE(g && v && nsteps >= 0 && (steps || nsteps == 0));
    API_BEGIN
    const NodeValues nv = node_values(*g->e, *v->v, std::vector<int>(steps, steps + nsteps));
    if (info) *info = gtob_node_info{nv.node, nv.kind, nv.player, nv.na};
    put(reach0, nv.reach[0]);
    put(reach1, nv.reach[1]);
    put(valid0, nv.valid[0]);
    put(valid1, nv.valid[1]);
    put(eq0, nv.eq[0]);
    put(eq1, nv.eq[1]);
    put(ev0, nv.ev[0]);
    put(ev1, nv.ev[1]);
    put(strategy, nv.strategy);
    put(action_ev, nv.action_ev);
    API_END
}
int gtob_gpu_runouts(gtob_gpu* g, const gtob_solver* v, const int* steps, int nsteps, gtob_runout_row* rows,
                     float* freqs, int max_rows, int max_actions, int* n_rows, int* player, int* num_actions,
                     double* pot) {
    REQUIRE(g && v && nsteps >= 0 && (steps || nsteps == 0) && rows && max_rows >= 0 && max_actions >= 0 && n_rows);
    API_BEGIN
    const Runouts r = runouts(*g->e, *v->v, std::vector<int>(steps, steps + nsteps));
    if ((int)r.rows.size() > max_rows)
        throw Error("invalid argument: " + std::to_string(r.rows.size()) + " runout rows, room for " +
                    std::to_string(max_rows));
    if (freqs && r.na > max_actions)
        throw Error("invalid argument: " + std::to_string(r.na) + " actions, room for " + std::to_string(max_actions));
    for (size_t k = 0; k < r.rows.size(); k++) {
        rows[k].card = r.rows[k].card;
        rows[k].eq[0] = r.rows[k].eq[0];
        rows[k].eq[1] = r.rows[k].eq[1];
        rows[k].ev[0] = r.rows[k].ev[0];
        rows[k].ev[1] = r.rows[k].ev[1];
        if (freqs)
            for (size_t a = 0; a < r.rows[k].freqs.size(); a++) freqs[k * max_actions + a] = r.rows[k].freqs[a];
    }
    *n_rows = (int)r.rows.size();
    if (player) *player = r.player;
    if (num_actions) *num_actions = r.na;
    if (pot) *pot = r.pot;
    API_END
}
int gtob_gpu_exploit_values(gtob_gpu* g, const gtob_solver* v, const int* steps, int nsteps, int exploiter,
                            gtob_node_info* info, float* reach, float* valid, float* br_ev, float* cur_ev, float* gain,
                            float* br_strategy, float* action_ev, float* averages) {
    REQUIRE(g && v && nsteps >= 0 && (steps || nsteps == 0) && (exploiter == 0 || exploiter == 1));
    API_BEGIN
    const ExploitValues x = exploit_values(*g->e, *v->v, std::vector<int>(steps, steps + nsteps), exploiter);
    if (info) *info = gtob_node_info{x.node, x.kind, x.player, x.na};
    put(reach, x.reach);
    put(valid, x.valid);
    put(br_ev, x.br_ev);
    put(cur_ev, x.cur_ev);
    put(gain, x.gain);
    put(br_strategy, x.br_strategy);
    put(action_ev, x.action_ev);
    if (averages) std::memcpy(averages, x.avg, sizeof(x.avg));
    API_END
}
int gtob_solver_path_view(const gtob_solver* v, const int* steps, int nsteps, char* out, uint64_t cap,
                          uint64_t* needed) {
    REQUIRE(v && needed && nsteps >= 0 && (steps || nsteps == 0) && (out || cap == 0));
    API_BEGIN
    const std::string js = path_view_json(*v->v, std::vector<int>(steps, steps + nsteps));
    *needed = js.size() + 1;
    if (cap > 0) {
        const size_t k = std::min<size_t>(js.size(), (size_t)cap - 1);
        std::memcpy(out, js.data(), k);
        out[k] = 0;
    }
    API_END
}
int gtob_nccl_unique_id(unsigned char out[128]) {
    REQUIRE(out);
    API_BEGIN
    nccl_unique_id(out);
    API_END
}
int gtob_gpu_new_sharded(const gtob_solver* v, int fmt, int engine, int rank, int world, const unsigned char id[128],
                         gtob_gpu** out) {
    REQUIRE(v && id && out && world >= 1 && rank >= 0 && rank < world && fmt >= -1 && fmt <= 3 &&
            engine >= GTOB_ENGINE_FUSED && engine <= GTOB_ENGINE_STAGED_RIVER);
    *out = nullptr;
    API_BEGIN
    auto red = make_nccl_reducer(rank, world, id);
    *out = new gtob_gpu{std::make_unique<GpuEngine>(*v->v, fmt, engine, rank, world, red)};
    API_END
}
int gtob_gpu_new_sharded_host(const gtob_solver* v, int fmt, int engine, int rank, int world, gtob_reduce_fn fn,
                              void* user, gtob_gpu** out) {
    REQUIRE(v && fn && out && world >= 1 && rank >= 0 && rank < world && fmt >= -1 && fmt <= 3 &&
            engine >= GTOB_ENGINE_FUSED && engine <= GTOB_ENGINE_STAGED_RIVER);
    *out = nullptr;
    API_BEGIN
    auto red = make_callback_reducer(fn, user);
    *out = new gtob_gpu{std::make_unique<GpuEngine>(*v->v, fmt, engine, rank, world, red)};
    API_END
}
int gtob_shards_new(const gtob_solver* v, int fmt, int engine, int nshards, gtob_shards** out) {
    REQUIRE(v && out && nshards >= 1 && nshards <= 64 && fmt >= -1 && fmt <= 3 && engine >= GTOB_ENGINE_FUSED &&
            engine <= GTOB_ENGINE_STAGED_RIVER);
    *out = nullptr;
    API_BEGIN
    auto g = std::make_unique<gtob_shards>();
    const cudaError_t rc = cudaGetDevice(&g->device);
    if (rc != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(rc));
    auto x = std::make_shared<HostExchange>(nshards);
    for (int k = 0; k < nshards; k++)
        g->e.push_back(std::make_unique<GpuEngine>(*v->v, fmt, engine, k, nshards, make_host_reducer(x, k)));
    *out = g.release();
    API_END
}
int gtob_shards_iterate(gtob_shards* g, int n) {
    REQUIRE(g && n >= 0);
    API_BEGIN
    g->all([&](int k) { g->e[k]->iterate(n); g->e[k]->synchronize(); });
    API_END
}
int gtob_shards_exploitability(gtob_shards* g, const gtob_solver* v, double* chips) {
    REQUIRE(g && v && chips);
    API_BEGIN
    std::vector<double> r(g->e.size());
    g->all([&](int k) { r[k] = g->e[k]->exploitability(*v->v); });
    for (double x : r)
        if (!(x == r[0]) && !(std::isnan(x) && std::isnan(r[0]))) throw Error("shards disagree on the exploitability");
    *chips = r[0];
    API_END
}
int gtob_shards_export_arena(gtob_shards* g, int which, int p, float* out) {
    REQUIRE(g && out && which >= 0 && which <= 2 && (p == 0 || p == 1));
    API_BEGIN
    const Spot& sp = *g->e[0]->plan_spot();
    const Tree& t = sp.tree;
    const size_t len = t.data_size[p], nh = sp.hands[p].size();
    std::vector<std::vector<float>> img(g->e.size(), std::vector<float>(len));
    for (size_t k = 0; k < g->e.size(); k++) g->e[k]->export_arena(which, p, img[k].data());
    std::memset(out, 0, len * sizeof(float));
    for (uint32_t nd = 0; nd < t.size(); nd++) {
        if (t.kind[nd] != kAction || t.player[nd] != p) continue;
        for (size_t k = 0; k < g->e.size(); k++)
            if (g->e[k]->plan().node_sidx[nd] >= 0) {
                std::memcpy(out + t.data_off[nd], img[k].data() + t.data_off[nd], t.nchild[nd] * nh * sizeof(float));
                break;
            }
    }
    API_END
}
int gtob_shards_sync_to_cpu(gtob_shards* g, gtob_solver* v, int strategy_only) {
    REQUIRE(g && v);
    API_BEGIN
    for (auto& e : g->e) e->sync_to_cpu(*v->v, strategy_only != 0);  // each shard writes its own nodes
    API_END
}
void gtob_shards_free(gtob_shards* g) { delete g; }
int gtob_spot_batch_queue(gtob_spot* const* spots, int n, int use_iso, int tile, gtob_batch_segment* out, int cap,
                          int* nseg, uint64_t* ntickets, uint64_t* nrecords) {
    REQUIRE(spots && n > 0 && tile >= 1 && cap >= 0 && (out || cap == 0) && nseg && ntickets && nrecords);
    for (int i = 0; i < n; i++) REQUIRE(spots[i]);
    API_BEGIN
    std::vector<Plan> plans(n);
    std::vector<const Plan*> ptr;
    for (int i = 0; i < n; i++) {
        plans[i] = build_plan(*spots[i]->s, use_iso != 0, kFuseFolds);
        ptr.push_back(&plans[i]);
    }
    std::vector<BatchSegment> q;
    *ntickets = batch_queue(ptr, tile, q, nrecords);
    *nseg = (int)q.size();
    for (int k = 0; k < std::min<int>(cap, (int)q.size()); k++) {
        const BatchSegment& g = q[k];
        out[k] = gtob_batch_segment{g.first, g.start, g.count, g.need, g.spot, g.step, g.kind, g.p, g.tile};
    }
    API_END
}
int gtob_spot_shard_visited(const gtob_spot* sp, int use_iso, int shard, int nshards, uint8_t* visited) {
    REQUIRE(sp && visited && nshards >= 1 && shard >= 0 && shard < nshards);
    API_BEGIN
    const Plan P = build_plan(*sp->s, use_iso != 0, kFuseFolds, shard, nshards);
    for (size_t i = 0; i < P.node_cslot.size(); i++) visited[i] = P.node_cslot[i] != kNoSlot ? 1 : 0;
    API_END
}
int gtob_spot_dl_plan(const gtob_spot* sp, uint32_t* nodes, float* pot, float* stack, int cap, int* n,
                      uint8_t* visited) {
    REQUIRE(sp && n && cap >= 0);
    API_BEGIN
    const Plan P = build_plan(*sp->s, false, kFuseFolds, 0, 1, true);
    *n = (int)P.leaves.size();
    for (int i = 0; i < std::min(cap, (int)P.leaves.size()); i++) {
        if (nodes) nodes[i] = P.leaves[i].node;
        if (pot) pot[i] = P.leaves[i].pot;
        if (stack) stack[i] = P.leaves[i].stack;
    }
    if (visited)
        for (size_t i = 0; i < P.node_cslot.size(); i++) visited[i] = P.node_cslot[i] != kNoSlot ? 1 : 0;
    API_END
}
struct gtob_batch {
    std::vector<std::shared_ptr<Spot>> spots;
    std::vector<std::unique_ptr<gtob_solver>> solvers;  // empty entries when the batch keeps none
    std::vector<BatchRow> rows;
    BatchRunStats stats;  // of the last persistent run
    int storage = 0, algo = 0, fmt = -1, engine = GTOB_ENGINE_STAGED;
    bool use_iso = true;
};
int gtob_batch_new(gtob_spot* const* spots, int n, int storage, int algo, int use_iso, int fmt, int engine, int keep,
                   gtob_batch** out) {
    REQUIRE(spots && out && n > 0 && (storage == 0 || storage == 1) && algo >= 0 && algo <= 2 && fmt >= -1 &&
            fmt <= 3 && engine >= GTOB_ENGINE_FUSED && engine <= GTOB_ENGINE_STAGED_RIVER);
    *out = nullptr;
    for (int i = 0; i < n; i++) REQUIRE(spots[i]);
    API_BEGIN
    auto b = std::make_unique<gtob_batch>();
    for (int i = 0; i < n; i++) {
        b->spots.push_back(spots[i]->s);
        b->solvers.push_back(keep ? std::make_unique<gtob_solver>(gtob_solver{
                                        std::make_unique<HostSolver>(spots[i]->s, storage, algo, use_iso != 0)})
                                  : nullptr);
    }
    b->rows.resize(n);
    b->storage = storage;
    b->algo = algo;
    b->use_iso = use_iso != 0;
    b->fmt = fmt;
    b->engine = engine;
    *out = b.release();
    API_END
}
int gtob_batch_run(gtob_batch* b, uint32_t max_iterations, double target_pct, uint32_t check_every, int workers) {
    REQUIRE(b && check_every > 0 && workers > 0);
    API_BEGIN
    std::vector<HostSolver*> hs;
    for (auto& v : b->solvers) hs.push_back(v ? v->v.get() : nullptr);
    run_batch(b->spots, hs, b->storage, b->algo, b->use_iso, b->fmt, b->engine, max_iterations, target_pct,
              check_every, workers, b->rows);
    API_END
}
int gtob_batch_run_persistent(gtob_batch* b, uint32_t max_iterations, double target_pct, uint32_t check_every,
                              int window) {
    REQUIRE(b && check_every > 0 && window > 0);
    API_BEGIN
    std::vector<HostSolver*> hs;
    for (auto& v : b->solvers) hs.push_back(v ? v->v.get() : nullptr);
    run_batch_persistent(b->spots, hs, b->storage, b->algo, b->use_iso, b->fmt, max_iterations, target_pct,
                         check_every, window, b->rows, &b->stats);
    API_END
}
int gtob_batch_stats_get(const gtob_batch* b, gtob_batch_stats* out) {
    REQUIRE(b && out);
    out->launches = b->stats.launches;
    out->kernel_ms = b->stats.kernel_ms;
    out->tuned = b->stats.tuned;
    out->tile = b->stats.tile;
    out->ctas_per_sm = b->stats.ctas_per_sm;
    out->grid = b->stats.grid;
    return GTOB_OK;
}
int gtob_batch_size(const gtob_batch* b) { return b ? (int)b->solvers.size() : 0; }
int gtob_batch_row_get(const gtob_batch* b, int i, gtob_batch_row* out) {
    REQUIRE(b && out && i >= 0 && i < (int)b->rows.size());
    const BatchRow& r = b->rows[i];
    out->status = r.error.empty() ? GTOB_OK : classify(r.error);
    out->iterations = r.iterations;
    out->exploit_pct = r.exploit_pct;
    out->seconds = r.seconds;
    out->ev[0] = r.ev[0];
    out->ev[1] = r.ev[1];
    return GTOB_OK;
}
int gtob_batch_root_cfv(gtob_batch* b, int i, int p, float* out, int cap, int* n) {
    REQUIRE(b && n && (p == 0 || p == 1) && i >= 0 && i < (int)b->rows.size() && cap >= 0);
    API_BEGIN
    const std::vector<float>& v = b->rows[i].root_cfv[p];
    *n = (int)v.size();
    if (out) std::memcpy(out, v.data(), std::min<size_t>(v.size(), (size_t)cap) * sizeof(float));
    API_END
}
const char* gtob_batch_error(const gtob_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->rows.size()) return "";
    return b->rows[i].error.c_str();
}
gtob_solver* gtob_batch_solver(gtob_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->solvers.size() || !b->solvers[i]) return nullptr;
    return b->solvers[i].get();
}
void gtob_batch_free(gtob_batch* b) { delete b; }

int gtob_gpu_save(gtob_gpu* g, const gtob_solver* v, const char* path) {
    REQUIRE(g && v && path);
    API_BEGIN
    g->e->save(*v->v, path);
    API_END
}
int gtob_gpu_load(const char* path, int storage, int fmt, int engine, gtob_solver** solver_out, gtob_gpu** gpu_out) {
    REQUIRE(path && solver_out && gpu_out && (storage == 0 || storage == 1) && fmt >= -1 && fmt <= 3 &&
            engine >= GTOB_ENGINE_FUSED && engine <= GTOB_ENGINE_STAGED_RIVER);
    *solver_out = nullptr;
    *gpu_out = nullptr;
    API_BEGIN
    std::ifstream in(path, std::ios::binary);
    if (!in) throw Error(std::string("cannot open ") + path);
    auto host = HostSolver::load_header(in, storage);
    auto eng = std::make_unique<GpuEngine>(*host, fmt, engine);
    eng->load_arenas(in, *host);
    *solver_out = new gtob_solver{std::move(host)};
    *gpu_out = new gtob_gpu{std::move(eng)};
    API_END
}
int gtob_gpu_new(const gtob_solver* v, int fmt, gtob_gpu** out) { return gtob_gpu_new_ex(v, fmt, GTOB_ENGINE_STAGED, out); }
int gtob_gpu_new_ex(const gtob_solver* v, int fmt, int engine, gtob_gpu** out) {
    REQUIRE(v && out && fmt >= -1 && fmt <= 3 && engine >= GTOB_ENGINE_FUSED && engine <= GTOB_ENGINE_STAGED_RIVER);
    *out = nullptr;
    API_BEGIN
    *out = new gtob_gpu{std::make_unique<GpuEngine>(*v->v, fmt, engine)};
    API_END
}
void gtob_gpu_free(gtob_gpu* g) { delete g; }
int gtob_gpu_iterate(gtob_gpu* g, int n) {
    REQUIRE(g && n >= 0);
    API_BEGIN
    g->e->iterate(n);
    API_END
}
int gtob_gpu_iterate_profiled(gtob_gpu* g, gtob_profile* out) {
    REQUIRE(g && out);
    API_BEGIN
    Profile p = g->e->iterate_profiled();
    std::memcpy(out->ms, p.ms, sizeof(p.ms));
    std::memcpy(out->launches, p.launches, sizeof(p.launches));
    API_END
}
int gtob_gpu_exploitability(gtob_gpu* g, const gtob_solver* v, double* chips) {
    REQUIRE(g && v && chips);
    API_BEGIN
    *chips = g->e->exploitability(*v->v);
    API_END
}
int gtob_gpu_sync_to_cpu(gtob_gpu* g, gtob_solver* v) {
    REQUIRE(g && v);
    API_BEGIN
    g->e->sync_to_cpu(*v->v, false);
    API_END
}
int gtob_gpu_sync_strategy(gtob_gpu* g, gtob_solver* v) {
    REQUIRE(g && v);
    API_BEGIN
    g->e->sync_to_cpu(*v->v, true);
    API_END
}
int gtob_gpu_synchronize(gtob_gpu* g) {
    REQUIRE(g);
    API_BEGIN
    g->e->synchronize();
    API_END
}
int gtob_gpu_update_locks(gtob_gpu* g, const gtob_solver* v) {
    REQUIRE(g && v);
    API_BEGIN
    g->e->update_locks(*v->v);
    API_END
}
uint32_t gtob_gpu_iteration(const gtob_gpu* g) { return g ? g->e->iteration() : 0; }
int gtob_gpu_info_get(gtob_gpu* g, gtob_gpu_info* o) {
    REQUIRE(g && o);
    const Plan& P = g->e->plan();
    o->device_bytes = g->e->device_bytes();
    o->visited_nodes = P.num_visited;
    o->cfv_slots = P.n_cslots;
    o->reach_slots[0] = P.n_rslots[0];
    o->reach_slots[1] = P.n_rslots[1];
    o->device_action_nodes[0] = P.n_anodes[0];
    o->device_action_nodes[1] = P.n_anodes[1];
    o->visited_terminals = P.visited_terminals;
    o->num_levels = (uint32_t)P.num_levels;
    o->num_river_slots = P.num_slots;
    o->arena_format = g->e->format();
    o->iter_bytes = g->e->iter_bytes();
    o->upload_bytes = g->e->upload_bytes();
    o->river_programs = g->e->river_programs();
    API_BEGIN
    o->iteration_kernels = g->e->iteration_kernels();  // captures the iteration graph if it is not yet
    API_END
}
int gtob_gpu_root_cfv(gtob_gpu* g, int p, int mode, float* out) {
    REQUIRE(g && out && (p == 0 || p == 1) && (mode == 0 || mode == 1));
    API_BEGIN
    g->e->root_cfv(p, mode, out);
    API_END
}
int gtob_gpu_export_arena(gtob_gpu* g, int which, int p, float* out) {
    REQUIRE(g && out && which >= 0 && which <= 2 && (p == 0 || p == 1));
    API_BEGIN
    g->e->export_arena(which, p, out);
    API_END
}
int gtob_gpu_read_node_static(gtob_gpu* g, int which, uint32_t node, float* out, uint64_t out_len,
                              uint64_t* written) {
    REQUIRE(g && out && which >= 0 && which <= 2);
    API_BEGIN
    const size_t n = g->e->read_node_static(which, node, out, (size_t)out_len);
    if (written) *written = n;
    API_END
}
int gtob_set_device(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g_err = std::string("cuda: ") + cudaGetErrorString(e);
        return GTOB_ECUDA;
    }
    return GTOB_OK;
}
int gtob_gpu_time_iterations(gtob_gpu* g, int n, double* ms) {
    REQUIRE(g && ms && n >= 0);
    API_BEGIN
    *ms = g->e->time_iterations(n);
    API_END
}
int gtob_gpu_discounts(gtob_gpu* g, float* out3) {
    REQUIRE(g && out3);
    API_BEGIN
    g->e->discounts(out3);
    API_END
}

int gtob_net_new(int din, int dh, int nhidden, int dout, uint64_t seed, gtob_net** out) {
    REQUIRE(out && din > 0 && dh > 0 && nhidden > 0 && nhidden <= 8 && dout > 0);
    *out = nullptr;
    API_BEGIN
    LeafNetDims d;
    d.din = din;
    d.dh = dh;
    d.nhidden = nhidden;
    d.dout = dout;
    *out = new gtob_net{std::make_shared<LeafNet>(d, seed)};
    API_END
}
void gtob_net_free(gtob_net* n) { delete n; }
int gtob_net_get_params(gtob_net* n, int l, float* w, float* b) {
    REQUIRE(n && (w || b));
    API_BEGIN
    n->n->get_params(l, w, b);
    API_END
}
int gtob_net_set_params(gtob_net* n, int l, const float* w, const float* b) {
    REQUIRE(n && (w || b));
    API_BEGIN
    n->n->set_params(l, w, b);
    API_END
}
int gtob_net_get_grads(gtob_net* n, int l, float* w, float* b) {
    REQUIRE(n && (w || b));
    API_BEGIN
    n->n->get_grads(l, w, b);
    API_END
}
int gtob_net_forward(gtob_net* n, const float* x, int rows, float* y) {
    REQUIRE(n && x && y && rows >= 0);
    API_BEGIN
    n->n->forward_host(x, rows, y);
    API_END
}
int gtob_net_gradients(gtob_net* n, const float* x, const float* t, const float* mask, int rows, double* loss) {
    REQUIRE(n && x && t && mask && loss && rows > 0);
    API_BEGIN
    *loss = n->n->gradients_host(x, t, mask, rows);
    API_END
}
int gtob_net_train(gtob_net* n, const float* x, const float* t, const float* mask, int count, int epochs, int batch,
                   float lr, uint64_t seed, float* losses) {
    REQUIRE(n && x && t && mask && count > 0 && epochs > 0 && batch > 0 && batch % 128 == 0 && lr > 0.0f);
    API_BEGIN
    n->n->train_host(x, t, mask, count, epochs, batch, lr, seed, losses);
    API_END
}
int gtob_gpu_new_dl(const gtob_solver* v, gtob_net* net, int fmt, int engine, gtob_gpu** out) {
    REQUIRE(v && net && out && fmt >= -1 && fmt <= 3 && engine >= GTOB_ENGINE_FUSED && engine <= GTOB_ENGINE_STAGED_RIVER);
    *out = nullptr;
    API_BEGIN
    *out = new gtob_gpu{std::make_unique<GpuEngine>(*v->v, fmt, engine, net->n)};
    API_END
}
int gtob_gpu_leaves(gtob_gpu* g, uint32_t* nodes, float* pot, float* stack, int cap, int* n) {
    REQUIRE(g && n && cap >= 0);
    API_BEGIN
    const auto& L = g->e->plan().leaves;
    *n = (int)L.size();
    for (int i = 0; i < std::min(cap, (int)L.size()); i++) {
        if (nodes) nodes[i] = L[i].node;
        if (pot) pot[i] = L[i].pot;
        if (stack) stack[i] = L[i].stack;
    }
    API_END
}
int gtob_gpu_node_sweep(gtob_gpu* g, uint32_t node, int p, int mode, float* cfv, float* reach0, float* reach1) {
    REQUIRE(g && (p == 0 || p == 1) && (mode == 0 || mode == 1));
    API_BEGIN
    g->e->node_sweep_values(node, p, mode, cfv, reach0, reach1, nullptr, nullptr);
    API_END
}
int gtob_gpu_node_strategy(gtob_gpu* g, uint32_t node, float* out) {
    REQUIRE(g && out);
    API_BEGIN
    g->e->node_average_strategy(node, out);
    API_END
}
int gtob_gemm_time(int m, int n, int k, int reps, double* ms) {
    REQUIRE(ms && m > 0 && n > 0 && k > 0 && m % 128 == 0 && n % 128 == 0 && k % 64 == 0 && reps > 0);
    API_BEGIN
    *ms = gemm_time_ms(m, n, k, reps);
    API_END
}
int gtob_gemm_bf16(const uint16_t* a, const uint16_t* b, int m, int n, int k, float* c) {
    REQUIRE(a && b && c && m > 0 && n > 0 && k > 0 && m % 128 == 0 && n % 128 == 0 && k % 64 == 0);
    API_BEGIN
    struct Buf {
        void* p = nullptr;
        explicit Buf(size_t bytes) {
            const cudaError_t e = cudaMalloc(&p, bytes);
            if (e != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(e));
        }
        ~Buf() { cudaFree(p); }
    } da((size_t)m * k * 2), db((size_t)n * k * 2), dc((size_t)m * n * 4), derr(4);
    auto ok = [](cudaError_t e) {
        if (e != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(e));
    };
    ok(cudaMemcpy(da.p, a, (size_t)m * k * 2, cudaMemcpyHostToDevice));
    ok(cudaMemcpy(db.p, b, (size_t)n * k * 2, cudaMemcpyHostToDevice));
    ok(cudaMemset(derr.p, 0, 4));
    GemmEpilogue e;
    e.out_f32 = (float*)dc.p;
    e.ld_f32 = n;
    gemm_bf16_tn((const __nv_bfloat16*)da.p, (const __nv_bfloat16*)db.p, m, n, k, e, (unsigned*)derr.p, nullptr);
    ok(cudaDeviceSynchronize());
    unsigned err = 0;
    ok(cudaMemcpy(&err, derr.p, 4, cudaMemcpyDeviceToHost));
    if (err) throw Error("timeout: a tensor-core matrix product's wait gave up");
    ok(cudaMemcpy(c, dc.p, (size_t)m * n * 4, cudaMemcpyDeviceToHost));
    API_END
}

}  // extern "C"
