// Device plan: a spot's tree flattened into level-ordered work items for the
// level-synchronous sweeps (the role of the reference's gpu/plan.rs), laid out
// for the B200 engine:
//   * every work item carries the indices its kernel needs (no per-node
//     pointer chasing on the device);
//   * reach and counterfactual-value vectors live in COMPACT slots: children
//     of one node get consecutive slots, and a node's reach for a player is
//     stored only where it changes (its "owner" slot);
//   * showdown rank tables are precomputed per river board so the terminal
//     evaluator is a strength-sorted prefix scan with card-removal
//     corrections and no searches on the device;
//   * each action node's arena block is hand-major ([hand * na + action]) and
//     starts on a 16-element boundary (32 B for 16-bit arenas, 64 B for f32).
#pragma once
#include <cstdint>
#include <vector>

#include "core.hpp"

namespace gtob {

constexpr int kArenaAlign = 16;  // elements

struct ActItem {           // one action node
    uint32_t node;         // tree node id (lock table index)
    uint32_t cslot;        // this node's cfv slot
    uint32_t child_cslot;  // first child's cfv slot (children consecutive)
    uint32_t rslot;        // actor's reach slot at this node
    uint32_t child_rslot;  // first child's actor reach slot (consecutive)
    uint32_t sidx;         // per-player compact index (per-node arena scales)
    uint64_t aoff;         // device arena offset (elements) in the actor's arena
    uint32_t actor;
    uint32_t na;
};
struct EdgeItem {  // one representative chance edge
    uint32_t prs[2];  // parent reach slots
    uint32_t crs[2];  // child reach slots
    uint32_t card;
    uint32_t pad;
};
struct FoldItem {
    uint32_t cslot;
    uint32_t rs[2];  // reach slots (the opponent's is read)
    uint32_t folder;
    float twin, tlose;
};
struct ShowItem {
    uint32_t cslot;
    uint32_t rs[2];
    uint32_t slot;  // dense river slot
    float twin, tlose, ttie;
    uint32_t pad;
};
struct ChanceItem {
    uint32_t cslot;
    uint32_t cc_start, cc_count;
    float inv;  // 1 / (46 - street), f32 as the reference computes it
};
struct CardEntry {  // chance card table (plan.rs:51-61)
    uint32_t card;
    uint32_t child_cslot;  // cfv slot of the orbit representative's child
    uint32_t perm;         // suit permutation index mapping card -> representative
    uint32_t pad;
};
// Per river slot and traverser: one entry per surviving hand, ranks relative
// to the opponent's strength-sorted list for the same board.
struct RankEntry {
    uint16_t idx;        // my hand index
    uint16_t lb, ub;     // #opp hands strictly weaker / not stronger
    uint16_t c1lo, c1hi; // #opp hands holding my card c1 among the first lb / ub
    uint16_t c2lo, c2hi; // same for c2
    uint16_t pad;
};

struct Span { uint32_t start, count; };

struct Plan {
    int num_levels = 0;
    int nh[2] = {0, 0};
    int nh_max = 0;
    bool iso_active = false;
    uint64_t num_visited = 0;
    // level-ordered work lists and per-level spans
    std::vector<ActItem> act;
    std::vector<Span> act_span;
    std::vector<EdgeItem> edge;
    std::vector<Span> edge_span;
    std::vector<FoldItem> fold;
    std::vector<Span> fold_span;
    std::vector<ShowItem> show;
    std::vector<Span> show_span;
    std::vector<ChanceItem> chance;
    std::vector<Span> chance_span;
    std::vector<CardEntry> cards;
    // slot counts
    uint64_t n_cslots = 0;
    uint64_t n_rslots[2] = {0, 0};
    // device arenas (per player)
    uint64_t arena_len[2] = {0, 0};  // elements incl. padding
    uint64_t n_anodes[2] = {0, 0};   // action nodes of the player on the device
    std::vector<uint32_t> anode_id[2];   // by sidx: tree node id
    std::vector<uint64_t> anode_off[2];  // by sidx: device offset
    // node -> action-item index (or -1) for locks
    std::vector<int32_t> node_sidx;  // per tree node: sidx within its actor's list, -1 if not on device
    // river slots
    uint32_t num_slots = 0;
    std::vector<uint32_t> slot_key;
    // per player q and slot: opponent-side tables (q as the OPPONENT)
    std::vector<uint32_t> sorted_off[2];   // [slot] -> start in sorted_idx
    std::vector<uint32_t> sorted_cnt[2];
    std::vector<uint16_t> sorted_idx[2];   // hand indices in ascending strength
    std::vector<uint32_t> ccard_off[2];    // [slot*53 + c] -> start in ccard_pos
    std::vector<uint16_t> ccard_pos[2];    // positions (in sorted order) of hands holding card c
    // per player p as TRAVERSER: rank entries per slot
    std::vector<uint32_t> rank_off[2];
    std::vector<uint32_t> rank_cnt[2];
    std::vector<RankEntry> rank[2];
    uint32_t max_sorted = 0;  // max opp list length over slots and players
    // per-hand tables
    std::vector<uint32_t> hcard_off[2];  // 53 offsets: hands of player q holding card c
    std::vector<uint16_t> hcard_idx[2];
    // algorithmic traffic model (elements / nodes visited per sweep)
    uint64_t visited_action_elems[2] = {0, 0};  // sum over device action nodes of na * nh
    uint64_t visited_terminals = 0;
};

Plan build_plan(const Spot& spot, bool use_iso);

}  // namespace gtob
