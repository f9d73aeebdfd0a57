// Device plan builder: see plan.hpp.  Traversal and orbit folding follow the
// reference's gpu/plan.rs:100-198 (levels = depth, representative chance
// branches only, card -> (representative, suit permutation) tables).
#include "plan.hpp"

#include <algorithm>
#include <cstring>
#include <atomic>
#include <exception>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <unordered_set>

namespace gtob {

namespace {
struct Visit {
    uint32_t node, level;
    uint8_t dealt[2];
    int ndealt;
    uint32_t cslot;
    uint32_t rs[2];
    uint32_t slot;  // river slot once the board is complete, else kNoSlot
    uint8_t from_chance;  // the node's parent deals a card (or it is a river spot's root)
};
bool is_terminal(uint8_t k) { return k == kFold || k == kShowdown; }

// Ids a subtree builder hands out before the merge knows its bases: kLocal + k.
constexpr uint32_t kLocal = 0x40000000u;
inline bool is_local(uint32_t x) { return x != kNoSlot && (x & 0xC0000000u) == kLocal; }

template <class T>
using Levels = std::vector<std::vector<std::pair<uint32_t, T>>>;

// One depth-first traversal over representative branches (plan.rs:100-198).
// The root builder covers the tree above the chance nodes and hands each
// representative chance child to a subtree builder (a task); subtree
// builders run on worker threads with ids of their own, which the merge
// offsets.
struct Builder {
    const Spot& sp;
    const Tree& t;
    Plan& P;
    std::vector<uint8_t>& visited;
    bool fused, fuse_folds, spawn;
    Levels<ActItem> act_l[4];  // by actor and river round: [2 * actor + in_river]
    Levels<EdgeItem> edge_l;
    Levels<FoldItem> fold_l;
    Levels<ShowItem> show_l[2];  // [in_river]: showdowns that end a river betting round
    Levels<ChanceItem> chance_l;
    std::vector<ChildRef> crefs;
    std::vector<TermInfo> terms;
    std::vector<CardEntry> cards;
    std::unordered_map<size_t, uint32_t> slot_of_key;
    std::vector<uint32_t> slot_key;
    uint32_t id0;  // first id: 1 for the root builder, kLocal for a subtree
    uint64_t next_c, next_r[2];
    uint64_t num_visited = 0, visited_terminals = 0;
    uint32_t max_children = 0;
    std::vector<uint32_t> nodes;  // the nodes visited (their slot entries are remapped at the merge)
    std::vector<Visit> tasks;     // root builder: the subtrees handed out
    std::vector<Visit> rroots;    // roots of river betting rounds (their visits)
    bool cut = false;             // root builder of a depth-limited plan
    std::vector<LeafItem> leaves;
    std::vector<uint32_t> cbase_of, rbase_of[2];

    Builder(const Spot& s, Plan& p, std::vector<uint8_t>& vis, bool fu, bool ff, bool root)
        : sp(s), t(s.tree), P(p), visited(vis), fused(fu), fuse_folds(ff), spawn(root), id0(root ? 0u : kLocal) {
        next_c = root ? 1 : kLocal;
        next_r[0] = next_r[1] = root ? 1 : kLocal;
    }
    bool in_place(uint8_t kind) const { return kind == kFold ? fuse_folds : kind == kShowdown ? fused : false; }
    void grow(uint32_t lv) {
        if (edge_l.size() <= lv) {
            for (auto& x : act_l) x.resize(lv + 1);
            edge_l.resize(lv + 1);
            fold_l.resize(lv + 1);
            show_l[0].resize(lv + 1);
            show_l[1].resize(lv + 1);
            chance_l.resize(lv + 1);
        }
    }
    uint32_t river_slot(const uint8_t* dealt, int nd) {
        const size_t key = sp.river_key(dealt, nd);
        auto it = slot_of_key.find(key);
        if (it != slot_of_key.end()) return it->second;
        const uint32_t sl = id0 + (uint32_t)slot_key.size();
        slot_of_key[key] = sl;
        slot_key.push_back((uint32_t)key);
        return sl;
    }
    uint32_t term_of(uint32_t c, const uint8_t* dealt, int nd) {
        TermInfo ti{(float)t.twin[c], (float)t.tlose[c], (float)t.ttie[c], 0};
        ti.aux = t.kind[c] == kFold ? t.player[c] : river_slot(dealt, nd);
        terms.push_back(ti);
        visited_terminals++;
        num_visited++;
        return (uint32_t)(terms.size() - 1);
    }
    void run(const Visit& start) {
        std::vector<Visit> stack;
        stack.push_back(start);
        Visit kids[256];  // children of the node being visited (nchild is a u8)
        while (!stack.empty()) {
            Visit v = stack.back();
            stack.pop_back();
            const uint32_t nd = v.node;
            visited[nd] = 1;
            P.node_cslot[nd] = v.cslot;
            P.node_rs[0][nd] = v.rs[0];
            P.node_rs[1][nd] = v.rs[1];
            nodes.push_back(nd);
            grow(v.level);
            num_visited++;
            switch (t.kind[nd]) {
                case kAction: {
                    const int a = t.player[nd], na = t.nchild[nd];
                    ActItem it{};
                    it.node = nd;
                    it.cslot = v.cslot;
                    it.rslot = v.rs[a];
                    it.oslot = v.rs[1 - a];
                    it.actor = (uint32_t)a;
                    it.na = (uint32_t)na;
                    it.cref = (uint32_t)crefs.size();
                    max_children = std::max<uint32_t>(max_children, (uint32_t)na);
                    int nkids = 0;
                    for (int k = 0; k < na; k++) {
                        const uint32_t c = t.child(nd, k);
                        if (is_terminal(t.kind[c]) && in_place(t.kind[c])) {
                            uint32_t ti = term_of(c, v.dealt, v.ndealt);
                            // With folds in place but showdowns not (the staged and warp
                            // engines), a fold child still gets the actor's reach slot: the
                            // down sweep, which has the actor's strategy at hand, writes the
                            // folding player's reach there, and the parent's up kernel reads
                            // it instead of recomputing that strategy.
                            const uint32_t frs = (t.kind[c] == kFold && !fused) ? (uint32_t)next_r[a]++ : kNoSlot;
                            crefs.push_back({t.kind[c] == kFold ? kChildFold : kChildShow, kNoSlot, frs, ti});
                            it.nterm++;
                            continue;
                        }
                        Visit cv = v;
                        cv.node = c;
                        cv.level = v.level + 1;
                        cv.from_chance = 0;
                        cv.cslot = (uint32_t)next_c++;
                        cv.rs[a] = (uint32_t)next_r[a]++;
                        crefs.push_back({kChildNode, cv.cslot, cv.rs[a], kNoSlot});
                        kids[nkids++] = cv;
                    }
                    const int in_river = t.street[nd] == 2 ? 1 : 0;
                    if (in_river && v.from_chance) rroots.push_back(v);
                    act_l[2 * a + in_river][v.level].push_back({nd, it});
                    for (int k = nkids - 1; k >= 0; k--) stack.push_back(kids[k]);
                    break;
                }
                case kChance: {
                    if (cut && t.street[nd] == 1) {  // deals the turn: a leaf when betting follows
                        uint32_t first = kSentinel;
                        for (int c = 0; c < 52 && first == kSentinel; c++) first = t.children[t.child_start[nd] + c];
                        if (first != kSentinel && t.kind[first] == kAction) {
                            const double half = sp.config.tree.starting_pot / 2.0;
                            LeafItem lf{nd, v.cslot, {v.rs[0], v.rs[1]}, (float)(t.put0[nd] + t.put1[nd]),
                                        (float)(sp.config.tree.effective_stack - (t.put0[nd] - half)), v.level, 0};
                            leaves.push_back(lf);
                            break;
                        }
                    }
                    std::vector<int> valid = P.iso_active ? sp.perms_fixing(v.dealt, v.ndealt) : std::vector<int>{0};
                    struct CardRep { uint8_t card, rep; uint32_t perm; };
                    std::vector<CardRep> cr;
                    for (int c = 0; c < 52; c++) {
                        uint32_t ch = t.children[t.child_start[nd] + c];
                        bool dealt = false;
                        for (int i = 0; i < v.ndealt; i++) dealt = dealt || v.dealt[i] == c;
                        if (ch == kSentinel || dealt) continue;
                        uint8_t rep = (uint8_t)c;
                        uint32_t krep = 0;
                        for (int k : valid) {
                            uint8_t pc = card_permute((uint8_t)c, sp.perms[k]);
                            if (pc < rep) { rep = pc; krep = (uint32_t)k; }
                        }
                        cr.push_back({(uint8_t)c, rep, krep});
                    }
                    uint32_t rep_cslot[52], rep_term[52];
                    ChanceItem ci{};
                    ci.cslot = v.cslot;
                    ci.inv = 1.0f / (float)(46 - (int)t.street[nd]);
                    ci.rs[0] = v.rs[0];
                    ci.rs[1] = v.rs[1];
                    int nkids = 0;
                    for (auto& x : cr) {
                        if (x.card != x.rep) continue;
                        const uint32_t c = t.children[t.child_start[nd] + x.card];
                        uint8_t d2[2] = {v.ndealt > 0 ? v.dealt[0] : (uint8_t)0, 0};
                        d2[v.ndealt] = x.card;
                        if (fused && t.kind[c] == kShowdown) {
                            rep_term[x.card] = term_of(c, d2, v.ndealt + 1);
                            rep_cslot[x.card] = kNoSlot;
                            continue;
                        }
                        Visit cv = v;
                        cv.node = c;
                        cv.level = v.level + 1;
                        cv.from_chance = 1;
                        cv.dealt[0] = d2[0];
                        cv.dealt[1] = d2[1];
                        cv.ndealt = v.ndealt + 1;
                        cv.slot = sp.board.size() + (size_t)cv.ndealt == 5 ? river_slot(cv.dealt, cv.ndealt) : kNoSlot;
                        cv.cslot = (uint32_t)next_c++;
                        cv.rs[0] = (uint32_t)next_r[0]++;
                        cv.rs[1] = (uint32_t)next_r[1]++;
                        rep_cslot[x.card] = cv.cslot;
                        rep_term[x.card] = kNoSlot;
                        EdgeItem e{{v.rs[0], v.rs[1]}, {cv.rs[0], cv.rs[1]}, x.card, 0};
                        edge_l[v.level].push_back({c, e});
                        kids[nkids++] = cv;
                    }
                    ci.cc_start = (uint32_t)cards.size();
                    ci.cc_count = (uint32_t)cr.size();
                    for (auto& x : cr) {
                        // low byte: the dealt card; second byte: its orbit representative
                        cards.push_back({(uint32_t)x.card | ((uint32_t)x.rep << 8), rep_cslot[x.rep], x.perm, rep_term[x.rep]});
                        if (rep_term[x.rep] != kNoSlot) ci.nterm++;
                    }
                    chance_l[v.level].push_back({nd, ci});
                    if (spawn) {  // each representative subtree becomes a task
                        for (int k = 0; k < nkids; k++) tasks.push_back(kids[k]);
                    } else {
                        for (int k = nkids - 1; k >= 0; k--) stack.push_back(kids[k]);
                    }
                    break;
                }
                case kFold: {
                    FoldItem f{v.cslot, {v.rs[0], v.rs[1]}, t.player[nd], (float)t.twin[nd], (float)t.tlose[nd]};
                    fold_l[v.level].push_back({nd, f});
                    visited_terminals++;
                    break;
                }
                default: {
                    ShowItem si{v.cslot, {v.rs[0], v.rs[1]}, v.slot != kNoSlot ? v.slot : river_slot(v.dealt, v.ndealt),
                                (float)t.twin[nd], (float)t.tlose[nd], (float)t.ttie[nd], 0};
                    show_l[!v.from_chance && t.street[nd] == 2 ? 1 : 0][v.level].push_back({nd, si});
                    visited_terminals++;
                    break;
                }
            }
        }
    }
};

// Where each builder's level lists go in a flat array: level by level, the
// builders in order (the groups, e.g. actors, one after another within a
// level).  off[g][lv][b] = start of builder b's group-g list of level lv.
struct FlatLayout {
    std::vector<std::vector<std::vector<size_t>>> off;
    std::vector<Span> span;                // per level
    std::vector<std::vector<Span>> gspan;  // per group, per level
    size_t total = 0;
};
template <class T>
FlatLayout flat_layout(size_t levels, const std::vector<std::vector<const Levels<T>*>>& lists) {
    // lists[b][g]: builder b's group-g levels
    const size_t nb = lists.size(), ng = nb ? lists[0].size() : 0;
    FlatLayout L;
    L.off.assign(ng, std::vector<std::vector<size_t>>(levels, std::vector<size_t>(nb, 0)));
    L.gspan.assign(ng, {});
    for (size_t lv = 0; lv < levels; lv++) {
        const size_t l0 = L.total;
        for (size_t g = 0; g < ng; g++) {
            const size_t g0 = L.total;
            for (size_t b = 0; b < nb; b++) {
                L.off[g][lv][b] = L.total;
                const Levels<T>& ls = *lists[b][g];
                if (lv < ls.size()) L.total += ls[lv].size();
            }
            L.gspan[g].push_back({(uint32_t)g0, (uint32_t)(L.total - g0)});
        }
        L.span.push_back({(uint32_t)l0, (uint32_t)(L.total - l0)});
    }
    return L;
}
template <class T, class V>
void flat_copy(const FlatLayout& L, size_t b, size_t g, Levels<T>& ls, V& flat) {
    for (size_t lv = 0; lv < ls.size(); lv++) {
        size_t o = L.off[g][lv][b];
        for (auto& x : ls[lv]) flat[o++] = x.second;
        std::vector<std::pair<uint32_t, T>>().swap(ls[lv]);
    }
}
// River programs (plan.hpp): one depth-first step list per river betting
// round.  P.river stays false, and the level sweeps keep these nodes, when a
// round does not fit the river kernel (an action node with more than kSKA
// actions, deeper than kRiverMaxDepth, or players not alternating from OOP).
constexpr int kRiverMaxActions = 4;
void build_river_programs(const Spot& sp, Plan& P, std::vector<Visit>& roots, unsigned threads) {
    const Tree& t = sp.tree;
    const size_t n = roots.size();
    if (!n) return;
    std::vector<std::vector<RStep>> prog(n);
    std::vector<uint32_t> depth(n, 0);
    std::atomic<bool> ok{true};
    parallel_for((n + 255) / 256, [&](size_t c) {
        struct Fr { uint32_t node; uint32_t depth, k, next; };
        std::vector<Fr> st;
        for (size_t r = c * 256; r < std::min(n, (c + 1) * 256); r++) {
            std::vector<RStep>& out = prog[r];
            auto node_step = [&](uint8_t op, uint32_t nd, uint32_t d, uint32_t k) {
                const int a = t.player[nd], na = t.nchild[nd];
                if (na > kRiverMaxActions || d >= (uint32_t)kRiverMaxDepth || a != (int)(d & 1) ||
                    t.kind[nd] != kAction || P.node_sidx[nd] < 0)
                    ok = false;
                RStep x{};
                x.op = op;
                x.depth = (uint8_t)d;
                x.k = (uint8_t)k;
                x.x = (uint8_t)(na | a << 7);
                x.sidx = (uint32_t)std::max(P.node_sidx[nd], 0);
                x.aoff = P.node_sidx[nd] >= 0 ? P.anode_off[a][P.node_sidx[nd]] : 0;
                out.push_back(x);
            };
            st.clear();
            node_step(kREnter, roots[r].node, 0, 0);
            st.push_back({roots[r].node, 0, 0, 0});
            while (!st.empty() && ok) {
                Fr& f = st.back();
                if (f.next < t.nchild[f.node]) {
                    const uint32_t j = f.next++;
                    const uint32_t ch = t.child(f.node, (int)j);
                    const uint32_t d = f.depth;
                    if (t.kind[ch] == kFold || t.kind[ch] == kShowdown) {
                        RStep x{};
                        x.op = t.kind[ch] == kFold ? kRFold : kRShow;
                        x.depth = (uint8_t)d;
                        x.k = (uint8_t)j;
                        x.x = t.kind[ch] == kFold ? t.player[ch] : 0;
                        const float tw = (float)t.twin[ch];
                        std::memcpy(&x.sidx, &tw, 4);
                        x.pay[0] = (float)t.tlose[ch];
                        x.pay[1] = (float)t.ttie[ch];
                        out.push_back(x);
                    } else if (t.kind[ch] == kAction) {
                        node_step(kREnter, ch, d + 1, j);
                        depth[r] = std::max(depth[r], d + 1);
                        st.push_back({ch, d + 1, j, 0});
                    } else {
                        ok = false;  // a chance node inside a river round
                    }
                } else {
                    node_step(kRExit, f.node, f.depth, f.k);
                    st.pop_back();
                }
            }
        }
    }, threads);
    if (!ok) return;
    std::vector<uint32_t> order(n);
    for (size_t r = 0; r < n; r++) order[r] = (uint32_t)r;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return prog[a].size() > prog[b].size(); });
    size_t total = 0;
    P.rtrees.resize(n);
    for (size_t i = 0; i < n; i++) {
        const uint32_t r = order[i];
        const Visit& v = roots[r];
        P.rtrees[i] = RTree{(uint32_t)total, (uint32_t)prog[r].size(), {v.rs[0], v.rs[1]}, v.cslot, v.slot, v.node,
                            depth[r]};
        total += prog[r].size();
        P.river_depth = std::max<int>(P.river_depth, (int)depth[r]);
    }
    P.rsteps.resize(total);
    parallel_for((n + 1023) / 1024, [&](size_t c) {
        for (size_t i = c * 1024; i < std::min(n, (c + 1) * 1024); i++)
            std::copy(prog[order[i]].begin(), prog[order[i]].end(), P.rsteps.begin() + P.rtrees[i].step_start);
    }, threads);
    P.river = true;
}
}  // namespace

Plan build_plan(const Spot& sp, bool use_iso, int fuse_mode, int shard, int nshards, bool cut_turn, bool river) {
    if (nshards < 1 || shard < 0 || shard >= nshards) throw Error("invalid argument: shard");
    if (cut_turn && (nshards > 1 || sp.tree.root_street != 0))
        throw Error("invalid argument: a depth-limited plan needs a flop spot and one shard");
    if (nshards > 1 && fuse_mode == kFuseAll)
        throw Error("sharding needs showdowns with slots of their own (not the fused engine)");
    const Tree& t = sp.tree;
    Plan P;
    const bool fused = fuse_mode == kFuseAll;
    P.fused = fused;
    P.fuse_folds = fuse_mode != kFuseNone;
    P.nh[0] = (int)sp.hands[0].size();
    P.nh[1] = (int)sp.hands[1].size();
    P.nh_max = std::max(P.nh[0], P.nh[1]);
    P.iso_active = use_iso && sp.perms.size() > 1;
    const size_t n = t.size();
    std::vector<uint8_t> visited(n, 0);
    P.node_cslot.assign(n, kNoSlot);
    P.node_rs[0].assign(n, kNoSlot);
    P.node_rs[1].assign(n, kNoSlot);

    // the tree above the chance nodes, then every representative chance
    // subtree on the worker threads
    Builder root(sp, P, visited, fused, P.fuse_folds, true);
    root.cut = cut_turn;
    P.cut_turn = cut_turn;
    const bool full_board = sp.board.size() == 5;
    root.run({0, 0, {0, 0}, 0, 0, {0, 0}, full_board ? root.river_slot(nullptr, 0) : kNoSlot,
              (uint8_t)(t.root_street == 2 ? 1 : 0)});
    P.shard = shard;
    P.nshards = nshards;
    // Sharded: this shard's representative subtrees, and the root builder's
    // cfv slots renumbered so that the children of each level's top chance
    // nodes take one contiguous run, ordered by the shard that computes them:
    // one sum over the shards per level, after zeroing the runs of the others.
    std::vector<uint32_t> root_perm;  // root builder's cfv slot -> final (sharded plans)
    if (nshards > 1) {
        struct Kid { uint32_t lv, owner, task, cslot; };
        std::unordered_map<uint32_t, uint32_t> task_of;  // child cfv slot -> task index
        for (size_t i = 0; i < root.tasks.size(); i++) task_of[root.tasks[i].cslot] = (uint32_t)i;
        std::vector<Kid> kids;
        std::unordered_set<uint32_t> seen;
        for (size_t lv = 0; lv < root.chance_l.size(); lv++)
            for (auto& x : root.chance_l[lv])
                for (uint32_t k = x.second.cc_start; k < x.second.cc_start + x.second.cc_count; k++) {
                    const uint32_t cs = root.cards[k].child_cslot;
                    if (cs == kNoSlot || !seen.insert(cs).second) continue;
                    const uint32_t ti = task_of.at(cs);
                    kids.push_back({(uint32_t)lv, ti % (uint32_t)nshards, ti, cs});
                }
        std::sort(kids.begin(), kids.end(), [](const Kid& a, const Kid& b) {
            return a.lv != b.lv ? a.lv < b.lv : a.owner != b.owner ? a.owner < b.owner : a.task < b.task;
        });
        const uint32_t nroot = (uint32_t)root.next_c;
        root_perm.assign(nroot, kNoSlot);
        for (const Kid& k : kids) root_perm[k.cslot] = 0;  // marked: placed below
        uint32_t next = 0;
        for (uint32_t c = 0; c < nroot; c++)
            if (root_perm[c] == kNoSlot) root_perm[c] = next++;
        P.reduce_span.assign(root.chance_l.size(), Span{0, 0});
        P.own_span.assign(root.chance_l.size(), Span{0, 0});
        for (size_t j = 0; j < kids.size(); j++) {
            const Kid& k = kids[j];
            const uint32_t at = next + (uint32_t)j;
            root_perm[k.cslot] = at;
            Span& r = P.reduce_span[k.lv];
            if (!r.count) r.start = at;
            r.count++;
            if ((int)k.owner == shard) {
                Span& o = P.own_span[k.lv];
                if (!o.count) o.start = at;
                o.count++;
            }
        }
        for (size_t lv = 0; lv < P.own_span.size(); lv++)  // an empty run sits at the level's start
            if (!P.own_span[lv].count) P.own_span[lv].start = P.reduce_span[lv].start;
        std::vector<Visit> mine;
        for (size_t i = 0; i < root.tasks.size(); i++)
            if ((int)(i % (size_t)nshards) == shard) mine.push_back(root.tasks[i]);
        root.tasks.swap(mine);
    }
    std::vector<std::unique_ptr<Builder>> subs;
    for (size_t i = 0; i < root.tasks.size(); i++)
        subs.push_back(std::make_unique<Builder>(sp, P, visited, fused, P.fuse_folds, false));
    // small trees (a few hundred thousand nodes) build faster on one thread,
    // and a batch builds several at once
    const unsigned threads = n >= (size_t(1) << 20) ? 16u : 1u;
    parallel_for(subs.size(), [&](size_t i) { subs[i]->run(root.tasks[i]); }, threads);
    // merge: river slots in first-visit order, then each subtree's ids offset
    // by what the builders before it handed out
    P.slot_key = root.slot_key;
    std::unordered_map<size_t, uint32_t> slot_of_key;
    for (size_t k = 0; k < root.slot_key.size(); k++) slot_of_key[root.slot_key[k]] = (uint32_t)k;
    struct Bases { uint32_t c, r[2], cref, term, card; std::vector<uint32_t> slot; };
    std::vector<Bases> bases(subs.size());
    uint64_t nc = root.next_c, nr[2] = {root.next_r[0], root.next_r[1]};
    size_t ncref = root.crefs.size(), nterm = root.terms.size(), ncard = root.cards.size();
    for (size_t i = 0; i < subs.size(); i++) {
        Builder& b = *subs[i];
        Bases& B = bases[i];
        B.c = (uint32_t)nc;
        B.r[0] = (uint32_t)nr[0];
        B.r[1] = (uint32_t)nr[1];
        B.cref = (uint32_t)ncref;
        B.term = (uint32_t)nterm;
        B.card = (uint32_t)ncard;
        nc += b.next_c - kLocal;
        nr[0] += b.next_r[0] - kLocal;
        nr[1] += b.next_r[1] - kLocal;
        ncref += b.crefs.size();
        nterm += b.terms.size();
        ncard += b.cards.size();
        for (uint32_t key : b.slot_key) {
            auto it = slot_of_key.find(key);
            if (it == slot_of_key.end()) {
                it = slot_of_key.emplace(key, (uint32_t)P.slot_key.size()).first;
                P.slot_key.push_back(key);
            }
            B.slot.push_back(it->second);
        }
    }
    if (nc >= kLocal || nr[0] >= kLocal || nr[1] >= kLocal) throw Error("tree too large for the plan's slot ids");
    std::vector<Builder*> bs{&root};
    for (auto& b : subs) bs.push_back(b.get());
    bases.insert(bases.begin(), Bases{0, {0, 0}, 0, 0, 0, {}});  // the root's ids are final
    size_t levels = 0;
    for (Builder* b : bs) levels = std::max(levels, b->edge_l.size());
    P.num_levels = (int)levels;
    auto layout_of = [&](auto member, int groups) {
        using L = std::remove_reference_t<decltype(member(*bs[0], 0))>;
        std::vector<std::vector<const L*>> lists(bs.size());
        for (size_t b = 0; b < bs.size(); b++)
            for (int g = 0; g < groups; g++) lists[b].push_back(&member(*bs[b], g));
        return flat_layout<typename L::value_type::value_type::second_type>(levels, lists);
    };
    const FlatLayout La = layout_of([](Builder& b, int g) -> Levels<ActItem>& { return b.act_l[g]; }, 4);
    const FlatLayout Le = layout_of([](Builder& b, int) -> Levels<EdgeItem>& { return b.edge_l; }, 1);
    const FlatLayout Lf = layout_of([](Builder& b, int) -> Levels<FoldItem>& { return b.fold_l; }, 1);
    const FlatLayout Ls = layout_of([](Builder& b, int g) -> Levels<ShowItem>& { return b.show_l[g]; }, 2);
    const FlatLayout Lc = layout_of([](Builder& b, int) -> Levels<ChanceItem>& { return b.chance_l; }, 1);
    P.act.resize(La.total);
    P.edge.resize(Le.total);
    P.fold.resize(Lf.total);
    P.show.resize(Ls.total);
    P.chance.resize(Lc.total);
    P.act_span = La.span;
    for (int a = 0; a < 2; a++) {  // groups [upper actor 0 | river actor 0 | upper actor 1 | river actor 1]
        P.act_span_upper[a] = La.gspan[2 * a];
        for (size_t lv = 0; lv < levels; lv++)
            P.act_span_actor[a].push_back(
                {La.gspan[2 * a][lv].start, La.gspan[2 * a][lv].count + La.gspan[2 * a + 1][lv].count});
    }
    P.edge_span = Le.span;
    P.fold_span = Lf.span;
    P.show_span = Ls.span;
    P.chance_span = Lc.span;
    P.crefs.resize(ncref);
    P.terms.resize(nterm);
    P.cards.resize(ncard);
    // each builder: its ids offset, then its lists copied into place
    parallel_for(bs.size(), [&](size_t i) {
        Builder& b = *bs[i];
        const Bases& B = bases[i];
        auto rc = [&](uint32_t& x) {
            if (is_local(x)) x = B.c + (x - kLocal);
            else if (x != kNoSlot && !root_perm.empty()) x = root_perm[x];  // a root builder's slot
        };
        auto rr = [&](uint32_t& x, int q) { if (is_local(x)) x = B.r[q] + (x - kLocal); };
        auto rs = [&](uint32_t& x) { if (is_local(x)) x = B.slot[x - kLocal]; };
        for (int g = 0; g < 4; g++)
            for (auto& lv : b.act_l[g])
                for (auto& x : lv) {
                    const int q = g >> 1;
                    ActItem& a = x.second;
                    for (uint32_t j = a.cref; j < a.cref + a.na; j++) {
                        ChildRef& cr = b.crefs[j];
                        rc(cr.cslot);
                        rr(cr.rslot, q);
                        if (cr.term != kNoSlot) cr.term += B.term;
                    }
                    rc(a.cslot);
                    rr(a.rslot, q);
                    rr(a.oslot, 1 - q);
                    a.cref += B.cref;
                }
        for (auto& lv : b.edge_l)
            for (auto& x : lv)
                for (int q = 0; q < 2; q++) {
                    rr(x.second.prs[q], q);
                    rr(x.second.crs[q], q);
                }
        for (auto& lv : b.fold_l)
            for (auto& x : lv) {
                rc(x.second.cslot);
                for (int q = 0; q < 2; q++) rr(x.second.rs[q], q);
            }
        for (auto& sl : b.show_l)
          for (auto& lv : sl)
            for (auto& x : lv) {
                rc(x.second.cslot);
                for (int q = 0; q < 2; q++) rr(x.second.rs[q], q);
                rs(x.second.slot);
            }
        for (auto& lv : b.chance_l)
            for (auto& x : lv) {
                rc(x.second.cslot);
                for (int q = 0; q < 2; q++) rr(x.second.rs[q], q);
                x.second.cc_start += B.card;
            }
        for (auto& ce : b.cards) {
            rc(ce.child_cslot);
            if (ce.term != kNoSlot) ce.term += B.term;
        }
        for (auto& ti : b.terms) rs(ti.aux);  // a showdown's slot; a fold's folding player stays
        for (auto& v : b.rroots) {
            rc(v.cslot);
            rr(v.rs[0], 0);
            rr(v.rs[1], 1);
            rs(v.slot);
        }
        for (uint32_t nd : b.nodes) {
            rc(P.node_cslot[nd]);
            rr(P.node_rs[0][nd], 0);
            rr(P.node_rs[1][nd], 1);
        }
        std::copy(b.crefs.begin(), b.crefs.end(), P.crefs.begin() + B.cref);
        std::copy(b.terms.begin(), b.terms.end(), P.terms.begin() + B.term);
        std::copy(b.cards.begin(), b.cards.end(), P.cards.begin() + B.card);
        std::vector<ChildRef>().swap(b.crefs);
        std::vector<TermInfo>().swap(b.terms);
        std::vector<CardEntry>().swap(b.cards);
        for (int g = 0; g < 4; g++) flat_copy(La, i, g, b.act_l[g], P.act);
        flat_copy(Le, i, 0, b.edge_l, P.edge);
        flat_copy(Lf, i, 0, b.fold_l, P.fold);
        flat_copy(Ls, i, 0, b.show_l[0], P.show);
        flat_copy(Ls, i, 1, b.show_l[1], P.show);
        flat_copy(Lc, i, 0, b.chance_l, P.chance);
    }, threads);
    for (Builder* b : bs) {
        P.num_visited += b->num_visited;
        P.visited_terminals += b->visited_terminals;
        P.max_children = std::max(P.max_children, b->max_children);
    }
    P.n_cslots = nc;
    P.leaves = std::move(root.leaves);  // the root builder's slots are final (depth-limited plans have one shard)
    if (nshards > 1) {  // the renumbered top part: the per-node slot table must follow it
        for (const ActItem& a : P.act)
            if (P.node_cslot[a.node] != a.cslot) throw Error("internal: a sharded plan's node slot table is stale");
    }
    P.n_rslots[0] = nr[0];
    P.n_rslots[1] = nr[1];

    // device arena layout: visited action nodes of each player in node order
    P.node_sidx.assign(n, -1);
    for (uint32_t nd = 0; nd < n; nd++) {
        if (!visited[nd] || t.kind[nd] != kAction) continue;
        int a = t.player[nd];
        uint64_t len = (uint64_t)t.nchild[nd] * P.nh[a];
        P.node_sidx[nd] = (int32_t)P.n_anodes[a];
        P.anode_id[a].push_back(nd);
        P.anode_off[a].push_back(P.arena_len[a]);
        P.n_anodes[a]++;
        P.arena_len[a] += (len + kArenaAlign - 1) / kArenaAlign * kArenaAlign;
        P.visited_action_elems[a] += len;
    }
    parallel_for((P.act.size() + 65535) / 65536, [&](size_t c) {
        for (size_t k = c * 65536; k < std::min(P.act.size(), (c + 1) * 65536); k++) {
            ActItem& x = P.act[k];
            x.sidx = (uint32_t)P.node_sidx[x.node];
            x.aoff = P.anode_off[x.actor][x.sidx];
        }
    }, threads);
    // showdowns of a level sorted by river slot and cut into batches of at
    // most kShowBatch with one slot each: a batch's CTA loads the slot's
    // tables once for all of them
    // (per level: the showdowns outside river rounds, then those inside)
    for (size_t l = 0; l < P.show_span.size(); l++) {
        const uint32_t b0 = (uint32_t)P.show_batch.size();
        for (int g = 0; g < 2; g++) {
            const Span s = Ls.gspan[g][l];
            auto first = P.show.begin() + s.start;
            {  // stable counting sort by slot
                std::vector<uint32_t> cnt(P.slot_key.size() + 1, 0);
                for (uint32_t k = 0; k < s.count; k++) cnt[first[k].slot + 1]++;
                for (size_t k = 1; k < cnt.size(); k++) cnt[k] += cnt[k - 1];
                std::vector<ShowItem> tmp(s.count);
                for (uint32_t k = 0; k < s.count; k++) tmp[cnt[first[k].slot]++] = first[k];
                std::copy(tmp.begin(), tmp.end(), first);
            }
            for (uint32_t k = 0; k < s.count;) {
                const uint32_t slot = P.show[s.start + k].slot;
                uint32_t e = k;
                while (e < s.count && e - k < (uint32_t)kShowBatch && P.show[s.start + e].slot == slot) e++;
                P.show_batch.push_back({s.start + k, e - k, slot, 0});
                k = e;
            }
            if (g == 0) P.show_batch_span_upper.push_back({b0, (uint32_t)P.show_batch.size() - b0});
        }
        P.show_batch_span.push_back({b0, (uint32_t)P.show_batch.size() - b0});
    }

    // per-hand card lists (fold evaluator: hands of player q holding card c)
    for (int q = 0; q < 2; q++) {
        std::vector<std::vector<uint16_t>> by(52);
        for (size_t i = 0; i < sp.hands[q].size(); i++) {
            by[sp.hands[q].c1[i]].push_back((uint16_t)i);
            by[sp.hands[q].c2[i]].push_back((uint16_t)i);
        }
        for (int c = 0; c < 52; c++) {
            P.hcard_off[q].push_back((uint32_t)P.hcard_idx[q].size());
            P.hcard_idx[q].insert(P.hcard_idx[q].end(), by[c].begin(), by[c].end());
        }
        P.hcard_off[q].push_back((uint32_t)P.hcard_idx[q].size());
    }

    // river slot tables
    P.num_slots = (uint32_t)P.slot_key.size();
    for (uint32_t s = 0; s < P.num_slots; s++) {
        const RiverBoard& rb = *sp.river.at(P.slot_key[s]);
        for (int q = 0; q < 2; q++) {
            P.sorted_off[q].push_back((uint32_t)P.sorted_idx[q].size());
            P.sorted_cnt[q].push_back((uint32_t)rb.idx[q].size());
            P.max_sorted = std::max<uint32_t>(P.max_sorted, (uint32_t)rb.idx[q].size());
            P.sorted_idx[q].insert(P.sorted_idx[q].end(), rb.idx[q].begin(), rb.idx[q].end());
            std::vector<std::vector<uint16_t>> by(52);
            for (size_t k = 0; k < rb.idx[q].size(); k++) {
                uint16_t h = rb.idx[q][k];
                by[sp.hands[q].c1[h]].push_back((uint16_t)k);
                by[sp.hands[q].c2[h]].push_back((uint16_t)k);
            }
            const size_t first = P.ccard_pos[q].size();
            P.bin_off[q].push_back((uint32_t)P.bin_start[q].size());
            P.bin_start[q].push_back(0);
            size_t bin_begin = 0;
            for (int c = 0; c < 52; c++) {
                P.ccard_off[q].push_back((uint32_t)P.ccard_pos[q].size());
                // close the bin if this card's whole list would not fit in it
                const size_t here = P.ccard_pos[q].size() - first;
                if (here - bin_begin + by[c].size() > 64) {
                    P.bin_start[q].push_back((uint16_t)here);
                    bin_begin = here;
                }
                P.ccard_pos[q].insert(P.ccard_pos[q].end(), by[c].begin(), by[c].end());
                P.ccard_card[q].insert(P.ccard_card[q].end(), by[c].size(), (uint8_t)c);
            }
            P.ccard_off[q].push_back((uint32_t)P.ccard_pos[q].size());
            const size_t total = P.ccard_pos[q].size() - first;
            if (total > bin_begin) P.bin_start[q].push_back((uint16_t)total);
            P.max_bins = std::max<uint32_t>(P.max_bins, (uint32_t)(P.bin_start[q].size() - P.bin_off[q].back() - 1));
        }
        for (int p = 0; p < 2; p++) {
            const int o = 1 - p;
            const auto& ms = rb.str[p];
            const auto& os = rb.str[o];
            const uint16_t* opos = P.ccard_pos[o].data();
            const uint32_t* ooff = P.ccard_off[o].data() + (size_t)s * 53;
            P.rank_off[p].push_back((uint32_t)P.rank[p].size());
            P.rank_cnt[p].push_back((uint32_t)ms.size());
            size_t lb = 0, ub = 0;
            for (size_t k = 0; k < ms.size(); k++) {
                while (lb < os.size() && os[lb] < ms[k]) lb++;
                if (ub < lb) ub = lb;
                while (ub < os.size() && os[ub] <= ms[k]) ub++;
                uint16_t h = rb.idx[p][k];
                RankEntry e{};
                e.idx = h;
                e.lb = (uint16_t)lb;
                e.ub = (uint16_t)ub;
                // Q index = segment base of the card + #entries of its list below the bound
                auto q_index = [&](int card, size_t bound) {
                    const uint16_t* b = opos + ooff[card];
                    const uint16_t* en = opos + ooff[card + 1];
                    const size_t base = (ooff[card] - ooff[0]) + (size_t)card;
                    return (uint16_t)(base + (std::lower_bound(b, en, (uint16_t)bound) - b));
                };
                const int h1 = sp.hands[p].c1[h], h2 = sp.hands[p].c2[h];
                e.q1lo = q_index(h1, lb);
                e.q1hi = q_index(h1, ub);
                e.q2lo = q_index(h2, lb);
                e.q2hi = q_index(h2, ub);
                e.cards = (uint16_t)(h1 | (h2 << 8));
                P.rank[p].push_back(e);
            }
            // my hands absent from this board's list (they hold a dealt card): value 0
            std::vector<uint8_t> on(P.nh[p], 0);
            for (uint16_t h : rb.idx[p]) on[h] = 1;
            P.zero_off[p].push_back((uint32_t)P.zero_idx[p].size());
            for (int h = 0; h < P.nh[p]; h++)
                if (!on[h]) P.zero_idx[p].push_back((uint16_t)h);
        }
    }
    for (int p = 0; p < 2; p++) {
        P.zero_off[p].push_back((uint32_t)P.zero_idx[p].size());
        P.bin_off[p].push_back((uint32_t)P.bin_start[p].size());
    }
    if (river && fuse_mode == kFuseFolds) {
        std::vector<Visit> roots;
        for (Builder* b : bs) roots.insert(roots.end(), b->rroots.begin(), b->rroots.end());
        build_river_programs(sp, P, roots, threads);
    }
    return P;
}

std::vector<std::vector<BatchSpan>> batch_steps(const Plan& P, int tile) {
    const int L = P.num_levels;
    std::vector<std::vector<BatchSpan>> st;
    auto add = [&](std::vector<BatchSpan> v) {
        std::vector<BatchSpan> keep;
        for (auto& x : v)
            if (x.s.count) keep.push_back(x);
        if (!keep.empty()) st.push_back(std::move(keep));
    };
    for (int p = 0; p < 2; p++) {
        std::vector<BatchSpan> first;
        if (p == 0) first.push_back({kBBegin, 0, {0, 1}, 1});
        first.push_back({kBRoot, 0, {0, 1}, 1});
        add(first);
        const int opp = 1 - p;
        for (int l = 0; l < L; l++)
            add({{kBDown, 0, P.act_span_actor[opp][l], tile}, {kBEdge, 1 << opp, P.edge_span[l], tile}});
        std::vector<BatchSpan> shows;
        for (int l = 0; l < L; l++) shows.push_back({kBShow, p, P.show_batch_span[l], 1});
        add(shows);
        for (int l = L - 1; l >= 0; l--)
            add({{kBChance, p, P.chance_span[l], tile},
                 {kBUpMine, p, P.act_span_actor[p][l], tile},
                 {kBUpOpp, p, P.act_span_actor[opp][l], tile}});
    }
    return st;
}

uint64_t batch_queue(const std::vector<const Plan*>& plans, int tile, std::vector<BatchSegment>& out,
                     uint64_t* records) {
    tile = std::max(1, std::min(tile, 64));
    std::vector<std::vector<std::vector<BatchSpan>>> steps(plans.size());
    size_t kmax = 0;
    for (size_t s = 0; s < plans.size(); s++) {
        steps[s] = batch_steps(*plans[s], tile);
        kmax = std::max(kmax, steps[s].size());
    }
    out.clear();
    std::vector<uint32_t> before(plans.size(), 0);  // tickets of the spot's steps so far
    uint64_t t = 0, rec = 0;
    for (size_t k = 0; k < kmax; k++)
        for (size_t s = 0; s < plans.size(); s++) {
            if (k >= steps[s].size()) continue;
            uint32_t here = 0;
            for (const BatchSpan& x : steps[s][k]) {
                const uint32_t nt = (x.s.count + (uint32_t)x.tile - 1) / (uint32_t)x.tile;
                out.push_back({t, x.s.start, x.s.count, before[s], (uint32_t)s, (uint32_t)k, x.kind, x.p, x.tile});
                t += nt;
                here += nt;
                rec += x.s.count;
            }
            before[s] += here;
        }
    if (records) *records = rec;
    return t;
}

}  // namespace gtob
