// Device plan: a spot's tree flattened into level-ordered work items for the
// level-synchronous sweeps (the role of the reference's gpu/plan.rs), laid out
// for the B200 engine:
//   * every work item carries the indices its kernel needs (no per-node
//     pointer chasing on the device); children are reached through ChildRef
//     entries holding their slots or, for terminals, their payoff record;
//   * reach and counterfactual-value vectors live in COMPACT slots, and a
//     node's reach for a player is stored only where it changes ("owner");
//   * in the fused layout terminals get no slots at all: the parent's up-sweep
//     kernel evaluates fold and showdown children in shared memory;
//   * showdown rank tables are precomputed per river board so the terminal
//     evaluator is a strength-sorted prefix scan with card-removal
//     corrections and no searches on the device;
//   * each action node's arena block is hand-major ([hand * na + action]) and
//     starts on a 16-element boundary (32 B for 16-bit arenas, 64 B for f32).
#pragma once
#include <algorithm>
#include <atomic>
#include <exception>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include <cstdint>
#include <vector>

#include "core.hpp"

namespace gtob {

constexpr int kArenaAlign = 16;  // elements
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

enum ChildKind : uint32_t { kChildNode = 0, kChildFold = 2, kChildShow = 3 };

struct ChildRef {
    uint32_t kind;   // kChildNode (has a cfv slot) or a terminal evaluated in place
    uint32_t cslot;  // cfv slot (kNoSlot for in-place terminals)
    uint32_t rslot;  // actor-side reach slot of the child (kNoSlot when not stored)
    uint32_t term;   // index into Plan::terms for terminals
};
struct TermInfo {
    float twin, tlose, ttie;
    uint32_t aux;  // fold: folding player; showdown: dense river slot
};
struct ActItem {       // one action node
    uint32_t node;     // tree node id
    uint32_t cslot;    // this node's cfv slot
    uint32_t rslot;    // actor's reach slot at this node
    uint32_t oslot;    // the other player's reach slot at this node
    uint32_t cref;     // first of na ChildRef entries
    uint32_t sidx;     // per-player compact index (per-node arena scales, locks)
    uint64_t aoff;     // device arena offset (elements) in the actor's arena
    uint32_t actor;
    uint32_t na;
    uint32_t nterm;    // terminal children (evaluated in place by the fused engine)
    uint32_t pad;
};
struct EdgeItem {  // one representative chance edge to a non-terminal child
    uint32_t prs[2];  // parent reach slots
    uint32_t crs[2];  // child reach slots
    uint32_t card;
    uint32_t pad;
};
struct FoldItem {
    uint32_t cslot;
    uint32_t rs[2];
    uint32_t folder;
    float twin, tlose;
};
struct alignas(16) ShowItem {
    uint32_t cslot;
    uint32_t rs[2];
    uint32_t slot;
    float twin, tlose, ttie;
    uint32_t pad;
};
struct ChanceItem {
    uint32_t cslot;
    uint32_t cc_start, cc_count;
    float inv;      // 1 / (46 - street), f32 as the reference computes it
    uint32_t rs[2]; // reach slots at the chance node (runout showdowns read them)
    uint32_t nterm; // card entries whose child is a showdown evaluated in place
    uint32_t pad;
};
struct CardEntry {  // chance card table (plan.rs:51-61)
    uint32_t card;         // dealt card | representative card << 8
    uint32_t child_cslot;  // cfv slot of the orbit representative's child (kNoSlot if in place)
    uint32_t perm;         // suit permutation index mapping card -> representative
    uint32_t term;         // representative showdown's TermInfo (runouts), else kNoSlot
};
// Per river slot and traverser: one entry per surviving hand, ranks relative
// to the opponent's strength-sorted list for the same board.
// The per-card prefixes of one board are stored concatenated: card c's
// segment starts at Q index qbase(c) = ccard_off[c] - ccard_off[0] + c and
// holds len(c) + 1 exclusive prefix values.
struct alignas(16) RankEntry {  // 16-byte aligned: one vector load on the device
    uint16_t idx;         // my hand index
    uint16_t lb, ub;      // #opp hands strictly weaker / not stronger
    uint16_t q1lo, q1hi;  // Q index of the prefix of card c1 over the first lb / ub opp hands
    uint16_t q2lo, q2hi;  // same for c2
    uint16_t cards;       // c1 | c2 << 8
};

struct Span { uint32_t start, count; };

// A depth-limited plan's leaf: a chance node dealing the turn below which
// the players still bet, cut from the tree; its values come from the turn
// leaf network each sweep (kind of an action node's child: kChildNode).
struct LeafItem {
    uint32_t node;    // tree node id of the chance node
    uint32_t cslot;   // its cfv slot
    uint32_t rs[2];   // reach slots at the node
    float pot, stack; // pot (both players' puts) and the remaining effective stack
    uint32_t level, pad;
};

// River subtree programs.  Every visited river betting round (an action node
// on the river whose parent deals the river, or the root of a river spot)
// is solved by one CTA walking the subtree depth first (cfr_river.cuh); its
// walk is a list of steps in pre-order, children in order:
//   kREnter  an action node: its depth, its index among its parent's children,
//            action count, actor, per-player compact index and arena offset;
//   kRExit   the same node once its last child is done (the same fields);
//   kRFold / kRShow  a terminal child of the node at `depth`: its index k and
//            payoffs (fold: the folding player in `x`).
enum RStepOp : uint8_t { kREnter = 0, kRExit = 1, kRFold = 2, kRShow = 3 };
struct alignas(16) RStep {
    uint8_t op, depth, k, x;  // x: na | actor << 7 (enter / exit), folding player (fold)
    uint32_t sidx;            // enter / exit: compact index; terminals: bits of twin
    union {
        uint64_t aoff;        // enter / exit: arena offset (elements) in the actor's arena
        float pay[2];         // terminals: tlose, ttie
    };
};
static_assert(sizeof(RStep) == 16, "RStep layout");
struct alignas(16) RTree {
    uint32_t step_start, step_count;
    uint32_t rs[2];  // both players' reach slots at the subtree root
    uint32_t cslot;  // the root's cfv slot (its value for the traverser goes there)
    uint32_t slot;   // the river board (dense river slot)
    uint32_t node;   // tree node id of the root
    uint32_t depth;  // deepest action node below the root (root = 0)
};
constexpr int kRiverMaxDepth = 8;  // river subtrees deeper than this keep the level sweeps

// Vectors of plain records whose resize does not zero them: the plan's flat
// tables are written in parallel right after they are sized, so the first
// touch of their pages happens on the worker threads.
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        if constexpr (sizeof...(A) == 0) ::new ((void*)p) U;
        else ::new ((void*)p) U(std::forward<A>(a)...);
    }
};
template <class T>
using PodVec = std::vector<T, NoInitAlloc<T>>;

// f(i) for i < n on up to max_threads (at most 16) host threads; the first
// exception is rethrown.
template <class F>
void parallel_for(size_t n, F f, unsigned max_threads = 16) {
    std::atomic<size_t> next{0};
    std::exception_ptr err;
    std::mutex mu;
    auto work = [&] {
        for (size_t i; (i = next.fetch_add(1)) < n;) {
            try {
                f(i);
            } catch (...) {
                std::lock_guard<std::mutex> lk(mu);
                if (!err) err = std::current_exception();
            }
        }
    };
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t nw = std::min<size_t>(n, std::max(1u, std::min({16u, max_threads, hw ? hw : 1u})));
    std::vector<std::thread> ts;
    for (size_t w = 1; w < nw; w++) ts.emplace_back(work);
    work();
    for (auto& th : ts) th.join();
    if (err) std::rethrow_exception(err);
}
constexpr int kShowBatch = 16;  // showdowns of one river slot evaluated by one CTA
struct ShowBatch {
    uint32_t start, count;  // a run of Plan::show (one level, one slot)
    uint32_t slot, pad;
};

// Which terminal children the parent's up-sweep kernel evaluates in place
// (no slots, no launches of their own).
enum FuseMode { kFuseNone = 0, kFuseFolds = 1, kFuseAll = 2 };

struct Plan {
    bool fused = false;       // showdown children evaluated in place too
    bool fuse_folds = false;  // fold children evaluated in place
    int num_levels = 0;
    int nh[2] = {0, 0};
    int nh_max = 0;
    bool iso_active = false;
    uint64_t num_visited = 0;
    PodVec<ActItem> act;
    std::vector<Span> act_span;
    std::vector<Span> act_span_actor[2];  // per level: the sub-span of each actor's nodes
    PodVec<EdgeItem> edge;
    std::vector<Span> edge_span;
    PodVec<FoldItem> fold;
    std::vector<Span> fold_span;
    PodVec<ShowItem> show;
    std::vector<Span> show_span;
    std::vector<ShowBatch> show_batch;      // per level, runs of same-slot showdowns
    std::vector<Span> show_batch_span;
    PodVec<ChanceItem> chance;
    std::vector<Span> chance_span;
    PodVec<CardEntry> cards;
    PodVec<ChildRef> crefs;
    PodVec<TermInfo> terms;
    uint32_t max_children = 0;  // over action nodes
    uint64_t n_cslots = 0;
    uint64_t n_rslots[2] = {0, 0};
    uint64_t arena_len[2] = {0, 0};
    uint64_t n_anodes[2] = {0, 0};
    std::vector<uint32_t> anode_id[2];
    std::vector<uint64_t> anode_off[2];
    std::vector<int32_t> node_sidx;
    // per tree node the sweep visits: its cfv slot and each player's reach
    // slot (kNoSlot for nodes it does not visit)
    std::vector<uint32_t> node_cslot, node_rs[2];
    int shard = 0, nshards = 1;
    bool cut_turn = false;         // depth-limited: the turn's betting chance nodes are leaves
    std::vector<LeafItem> leaves;  // (depth-limited plans)
    // per level, the contiguous cfv slots of the representative children of
    // that level's top chance nodes, which the shards split among them, and
    // the run of them this shard computes (the others it zeroes before each
    // sum); empty without sharding
    std::vector<Span> reduce_span, own_span;
    uint32_t num_slots = 0;
    std::vector<uint32_t> slot_key;
    std::vector<uint32_t> sorted_off[2];
    std::vector<uint32_t> sorted_cnt[2];
    std::vector<uint16_t> sorted_idx[2];
    std::vector<uint32_t> ccard_off[2];   // [slot*53 + c] -> start of card c's list in ccard_pos
    std::vector<uint16_t> ccard_pos[2];   // sorted-order positions of the opponent hands holding c
    std::vector<uint8_t> ccard_card[2];   // card of each ccard_pos entry
    // Card lists of one board packed, whole cards only, into bins of <= 64
    // entries (entry offsets relative to the slot's first entry).
    std::vector<uint32_t> bin_off[2];     // [slot] -> first entry in bin_start (num_slots + 1)
    std::vector<uint16_t> bin_start[2];   // nbins + 1 offsets per slot
    uint32_t max_bins = 0;
    std::vector<uint32_t> rank_off[2];
    std::vector<uint32_t> rank_cnt[2];
    std::vector<RankEntry> rank[2];
    std::vector<uint32_t> zero_off[2];  // [slot] -> start in zero_idx (num_slots + 1 entries)
    std::vector<uint16_t> zero_idx[2];  // my hands blocked by the board (cfv 0)
    uint32_t max_sorted = 0;
    std::vector<uint32_t> hcard_off[2];
    std::vector<uint16_t> hcard_idx[2];
    uint64_t visited_action_elems[2] = {0, 0};
    uint64_t visited_terminals = 0;
    // River programs (staged engine).  Action nodes and showdowns inside
    // river betting rounds sit after the other nodes of their level (within
    // each actor's run for action nodes); the *_upper spans leave them out,
    // and the river sweep solves them with one program per subtree instead.
    bool river = false;                        // programs built (every river subtree qualifies)
    std::vector<Span> act_span_upper[2];       // per level and actor: nodes outside river rounds
    std::vector<Span> show_batch_span_upper;   // per level: batches of showdowns outside river rounds
    std::vector<RTree> rtrees;                 // largest first
    PodVec<RStep> rsteps;
    int river_depth = 0;                       // deepest river action node (root = 0), over all programs
};

// The batched iteration's work queue (the persistent multi-spot kernel,
// kernels/cfr_batch.cuh).  A spot's CFR iteration is a list of steps in the
// order of the level sweeps' launches -- per traverser p = 0, 1: the
// iteration's discounts (p = 0 only) and the root reach; each level of the
// down sweep (the opponent's action nodes and the chance edges); the
// showdown batches of every level; each level of the up sweep, deepest
// first (chance nodes, the traverser's and the opponent's action nodes) --
// and a step is up to three spans of one kind of record (the staged engine's
// node records, chance edges, showdown batches, chance nodes).  Records of
// one step never depend on each other.
enum BatchKind : uint32_t { kBBegin = 0, kBRoot = 1, kBDown = 2, kBEdge = 3, kBShow = 4, kBChance = 5, kBUpMine = 6,
                            kBUpOpp = 7 };
struct BatchSpan {
    int kind, p;  // p: traverser (show, chance, up); edges: the players whose reach is refreshed (a mask)
    Span s;
    int tile;     // records per ticket
};
std::vector<std::vector<BatchSpan>> batch_steps(const Plan& P, int tile);
// One queue segment: a span of one step of one spot, cut into tickets of
// `tile` records.  Segments are ordered by step index, then spot, and a
// segment's `need` counts the tickets of its spot's earlier steps -- all of
// them numbered below the segment's first ticket, so a ticket only waits
// on lower tickets.
struct BatchSegment {
    uint64_t first;  // first ticket
    uint32_t start, count, need;
    uint32_t spot, step;
    int kind, p, tile;
};
// The queue of one batched iteration of the given plans; returns the ticket
// count (*records: the node records it covers).
uint64_t batch_queue(const std::vector<const Plan*>& plans, int tile, std::vector<BatchSegment>& out,
                     uint64_t* records);

// shard / nshards: the representative subtrees below the first chance nodes
// are dealt round-robin over nshards plans, each keeping the whole tree above
// them; the values of those subtrees' roots are summed over the shards
// (reduce_span: each is nonzero on one shard only) before the chance nodes
// above them add them up (a flop sharded by turn card).
// cut_turn: a depth-limited plan -- every chance node that deals the turn
// and leads to more betting becomes a leaf (Plan::leaves) instead of a
// subtree; all-in runouts stay exact.
// river: also build the river programs (fuse_mode kFuseFolds only).
Plan build_plan(const Spot& spot, bool use_iso, int fuse_mode, int shard = 0, int nshards = 1, bool cut_turn = false,
                bool river = false);

}  // namespace gtob
