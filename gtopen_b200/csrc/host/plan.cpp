// Device plan builder: see plan.hpp.  Traversal and orbit folding follow the
// reference's gpu/plan.rs:100-198 (levels = depth, representative chance
// branches only, card -> (representative, suit permutation) tables).
#include "plan.hpp"

#include <algorithm>
#include <unordered_map>

namespace gtob {

namespace {
struct Visit {
    uint32_t node, level;
    uint8_t dealt[2];
    int ndealt;
    uint32_t cslot;
    uint32_t rs[2];
    uint32_t slot;  // river slot once the board is complete, else kNoSlot
};
template <class T>
void flatten(std::vector<std::vector<std::pair<uint32_t, T>>>& by_level, std::vector<T>& flat, std::vector<Span>& span) {
    size_t total = 0;
    for (auto& lst : by_level) total += lst.size();
    flat.reserve(total);
    auto by_node = [](const auto& a, const auto& b) { return a.first < b.first; };
    for (auto& lst : by_level) {
        // the traversal visits a level's nodes in node order already; sort only if not
        if (!std::is_sorted(lst.begin(), lst.end(), by_node)) std::sort(lst.begin(), lst.end(), by_node);
        span.push_back({(uint32_t)flat.size(), (uint32_t)lst.size()});
        for (auto& x : lst) flat.push_back(x.second);
        std::vector<std::pair<uint32_t, T>>().swap(lst);
    }
}
bool is_terminal(uint8_t k) { return k == kFold || k == kShowdown; }
}  // namespace

Plan build_plan(const Spot& sp, bool use_iso, int fuse_mode) {
    const Tree& t = sp.tree;
    Plan P;
    const bool fused = fuse_mode == kFuseAll;
    P.fused = fused;
    P.fuse_folds = fuse_mode != kFuseNone;
    auto in_place = [&](uint8_t kind) { return kind == kFold ? P.fuse_folds : kind == kShowdown ? fused : false; };
    P.nh[0] = (int)sp.hands[0].size();
    P.nh[1] = (int)sp.hands[1].size();
    P.nh_max = std::max(P.nh[0], P.nh[1]);
    P.iso_active = use_iso && sp.perms.size() > 1;
    const size_t n = t.size();

    std::vector<std::vector<std::pair<uint32_t, ActItem>>> act_l;
    std::vector<std::vector<std::pair<uint32_t, EdgeItem>>> edge_l;
    std::vector<std::vector<std::pair<uint32_t, FoldItem>>> fold_l;
    std::vector<std::vector<std::pair<uint32_t, ShowItem>>> show_l;
    std::vector<std::vector<std::pair<uint32_t, ChanceItem>>> chance_l;
    auto grow = [&](uint32_t lv) {
        if (act_l.size() <= lv) {
            act_l.resize(lv + 1);
            edge_l.resize(lv + 1);
            fold_l.resize(lv + 1);
            show_l.resize(lv + 1);
            chance_l.resize(lv + 1);
        }
    };
    std::unordered_map<size_t, uint32_t> slot_of_key;
    auto river_slot = [&](const uint8_t* dealt, int nd) {
        size_t key = sp.river_key(dealt, nd);
        auto it = slot_of_key.find(key);
        if (it != slot_of_key.end()) return it->second;
        uint32_t s = (uint32_t)P.slot_key.size();
        slot_of_key[key] = s;
        P.slot_key.push_back((uint32_t)key);
        return s;
    };
    auto term_of = [&](uint32_t c, const uint8_t* dealt, int nd) {
        TermInfo ti{(float)t.twin[c], (float)t.tlose[c], (float)t.ttie[c], 0};
        ti.aux = t.kind[c] == kFold ? t.player[c] : river_slot(dealt, nd);
        P.terms.push_back(ti);
        P.visited_terminals++;
        P.num_visited++;
        return (uint32_t)(P.terms.size() - 1);
    };
    std::vector<uint8_t> visited(n, 0);
    P.node_cslot.assign(n, kNoSlot);
    P.node_rs[0].assign(n, kNoSlot);
    P.node_rs[1].assign(n, kNoSlot);
    {  // capacity for the flat tables (no regrowth during the traversal)
        size_t nchild = 0, nterm = 0;
        for (size_t i = 0; i < n; i++) {
            if (t.kind[i] == kAction) nchild += t.nchild[i];
            else if (is_terminal(t.kind[i])) nterm++;
        }
        P.crefs.reserve(nchild);
        P.terms.reserve(nterm);
    }

    uint64_t next_c = 1, next_r[2] = {1, 1};
    std::vector<Visit> stack;
    const bool full_board = sp.board.size() == 5;
    stack.push_back({0, 0, {0, 0}, 0, 0, {0, 0}, full_board ? river_slot(nullptr, 0) : kNoSlot});
    Visit kids[256];  // children of the node being visited (nchild is a u8)
    while (!stack.empty()) {
        Visit v = stack.back();
        stack.pop_back();
        const uint32_t nd = v.node;
        visited[nd] = 1;
        P.node_cslot[nd] = v.cslot;
        P.node_rs[0][nd] = v.rs[0];
        P.node_rs[1][nd] = v.rs[1];
        grow(v.level);
        P.num_visited++;
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
                it.cref = (uint32_t)P.crefs.size();
                P.max_children = std::max<uint32_t>(P.max_children, (uint32_t)na);
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
                        P.crefs.push_back({t.kind[c] == kFold ? kChildFold : kChildShow, kNoSlot, frs, ti});
                        it.nterm++;
                        continue;
                    }
                    Visit cv = v;
                    cv.node = c;
                    cv.level = v.level + 1;
                    cv.cslot = (uint32_t)next_c++;
                    cv.rs[a] = (uint32_t)next_r[a]++;
                    P.crefs.push_back({kChildNode, cv.cslot, cv.rs[a], kNoSlot});
                    kids[nkids++] = cv;
                }
                act_l[v.level].push_back({nd, it});
                for (int k = nkids - 1; k >= 0; k--) stack.push_back(kids[k]);
                break;
            }
            case kChance: {
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
                ci.cc_start = (uint32_t)P.cards.size();
                ci.cc_count = (uint32_t)cr.size();
                for (auto& x : cr) {
                    // low byte: the dealt card; second byte: its orbit representative
                    P.cards.push_back({(uint32_t)x.card | ((uint32_t)x.rep << 8), rep_cslot[x.rep], x.perm, rep_term[x.rep]});
                    if (rep_term[x.rep] != kNoSlot) ci.nterm++;
                }
                chance_l[v.level].push_back({nd, ci});
                for (int k = nkids - 1; k >= 0; k--) stack.push_back(kids[k]);
                break;
            }
            case kFold: {
                FoldItem f{v.cslot, {v.rs[0], v.rs[1]}, t.player[nd], (float)t.twin[nd], (float)t.tlose[nd]};
                fold_l[v.level].push_back({nd, f});
                P.visited_terminals++;
                break;
            }
            default: {
                ShowItem si{v.cslot, {v.rs[0], v.rs[1]}, v.slot != kNoSlot ? v.slot : river_slot(v.dealt, v.ndealt),
                            (float)t.twin[nd], (float)t.tlose[nd], (float)t.ttie[nd], 0};
                show_l[v.level].push_back({nd, si});
                P.visited_terminals++;
                break;
            }
        }
    }
    P.n_cslots = next_c;
    P.n_rslots[0] = next_r[0];
    P.n_rslots[1] = next_r[1];
    P.num_levels = (int)act_l.size();

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
    for (auto& lst : act_l)
        for (auto& x : lst) {
            int a = (int)x.second.actor;
            x.second.sidx = (uint32_t)P.node_sidx[x.first];
            x.second.aoff = P.anode_off[a][x.second.sidx];
        }
    flatten(act_l, P.act, P.act_span);
    // within a level, player 0's nodes first: a down sweep that only has to
    // refresh one player's reach launches over that player's sub-span
    for (size_t l = 0; l < P.act_span.size(); l++) {
        const Span s = P.act_span[l];
        auto first = P.act.begin() + s.start;
        auto mid = std::stable_partition(first, first + s.count, [](const ActItem& x) { return x.actor == 0; });
        const uint32_t n0 = (uint32_t)(mid - first);
        P.act_span_actor[0].push_back({s.start, n0});
        P.act_span_actor[1].push_back({s.start + n0, s.count - n0});
    }
    flatten(edge_l, P.edge, P.edge_span);
    flatten(fold_l, P.fold, P.fold_span);
    flatten(show_l, P.show, P.show_span);
    // showdowns of a level sorted by river slot and cut into batches of at
    // most kShowBatch with one slot each: a batch's CTA loads the slot's
    // tables once for all of them
    for (size_t l = 0; l < P.show_span.size(); l++) {
        const Span s = P.show_span[l];
        auto first = P.show.begin() + s.start;
        {  // stable counting sort by slot
            std::vector<uint32_t> cnt(P.slot_key.size() + 1, 0);
            for (uint32_t k = 0; k < s.count; k++) cnt[first[k].slot + 1]++;
            for (size_t k = 1; k < cnt.size(); k++) cnt[k] += cnt[k - 1];
            std::vector<ShowItem> tmp(s.count);
            for (uint32_t k = 0; k < s.count; k++) tmp[cnt[first[k].slot]++] = first[k];
            std::copy(tmp.begin(), tmp.end(), first);
        }
        const uint32_t b0 = (uint32_t)P.show_batch.size();
        for (uint32_t k = 0; k < s.count;) {
            const uint32_t slot = P.show[s.start + k].slot;
            uint32_t e = k;
            while (e < s.count && e - k < (uint32_t)kShowBatch && P.show[s.start + e].slot == slot) e++;
            P.show_batch.push_back({s.start + k, e - k, slot, 0});
            k = e;
        }
        P.show_batch_span.push_back({b0, (uint32_t)P.show_batch.size() - b0});
    }
    flatten(chance_l, P.chance, P.chance_span);

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
    return P;
}

}  // namespace gtob
