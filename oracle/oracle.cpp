// CPU oracle for the GTOpen postflop DCFR hot path -- TEST INFRASTRUCTURE.
//
// A plain C++ restatement of the reference CPU engine, used only by tests/,
// __graft_entry__.smoke() and the CPU-baseline leg of bench.py.  Every
// function cites the reference source it follows (paths inside the reference
// project).  Arithmetic follows the reference exactly: f32 vectors, f64
// terminal sweeps, reciprocal-then-multiply regret matching, round-ties-even
// saturating quantisation, f64 discount weights.  Build: oracle/Makefile.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <cfenv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static thread_local std::string g_err;
struct Err { std::string msg; };
[[noreturn]] static void fail(const std::string& m) { throw Err{m}; }

using Card = uint8_t;
static const uint32_t SENTINEL = 0xFFFFFFFFu;
static const char RANKS[] = "23456789TJQKA";
static const char SUITS[] = "cdhs";

// ---------------------------------------------------------------- cards.rs
static inline int rank_of(Card c) { return c >> 2; }
static inline int suit_of(Card c) { return c & 3; }
static inline Card make_card(int r, int s) { return (Card)((r << 2) | s); }
static inline uint64_t cmask(Card c) { return 1ull << c; }
static int rank_from_char(char ch) {  // cards.rs:37-40
    ch = (char)toupper((unsigned char)ch);
    for (int i = 0; i < 13; i++) if (RANKS[i] == ch) return i;
    return -1;
}
static int suit_from_char(char ch) {  // cards.rs:42-45
    ch = (char)tolower((unsigned char)ch);
    for (int i = 0; i < 4; i++) if (SUITS[i] == ch) return i;
    return -1;
}
static std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && isspace((unsigned char)s[a])) a++;
    while (b > a && isspace((unsigned char)s[b - 1])) b--;
    return s.substr(a, b - a);
}
static Card card_from_str(const std::string& s0) {  // cards.rs:47-55
    std::string s = trim(s0);
    if (s.size() != 2) fail("invalid card: " + s0);
    int r = rank_from_char(s[0]);
    if (r < 0) fail("invalid rank in card: " + s0);
    int su = suit_from_char(s[1]);
    if (su < 0) fail("invalid suit in card: " + s0);
    return make_card(r, su);
}
static std::vector<Card> parse_cards(const std::string& s) {  // cards.rs:66-86
    std::string cl;
    for (char c : s) if (!isspace((unsigned char)c) && c != ',') cl.push_back(c);
    if (cl.size() % 2) fail("invalid card list: " + s);
    std::vector<Card> out;
    uint64_t seen = 0;
    for (size_t i = 0; i < cl.size(); i += 2) {
        Card c = card_from_str(cl.substr(i, 2));
        if (seen & cmask(c)) fail("duplicate card in list: " + s);
        seen |= cmask(c);
        out.push_back(c);
    }
    return out;
}
static inline Card permute_card(Card c, const std::array<uint8_t, 4>& pm) {  // cards.rs:94
    return make_card(rank_of(c), pm[suit_of(c)]);
}
static inline int combo_index(Card a, Card b) {  // cards.rs:100-103
    int hi = a > b ? a : b, lo = a > b ? b : a;
    return hi * (hi - 1) / 2 + lo;
}
static inline void combo_from_index(int idx, Card* hi_out, Card* lo_out) {  // cards.rs:106-114
    int hi = 1;
    while ((hi + 1) * hi / 2 <= idx) hi++;
    *hi_out = (Card)hi;
    *lo_out = (Card)(idx - hi * (hi - 1) / 2);
}
static std::string card_str(Card c) { return std::string(1, RANKS[rank_of(c)]) + SUITS[suit_of(c)]; }

// canonical flops (cards.rs:261-311) and the systematic subset (cards.rs:236-259)
static std::vector<std::pair<std::string, uint32_t>> canonical_flops() {
    std::vector<std::array<uint8_t, 4>> perms;
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
            if (b == a) continue;
            for (int c = 0; c < 4; c++) {
                if (c == a || c == b) continue;
                perms.push_back({(uint8_t)a, (uint8_t)b, (uint8_t)c, (uint8_t)(6 - a - b - c)});
            }
        }
    std::map<std::array<uint8_t, 3>, uint32_t> classes;
    for (int x = 0; x < 52; x++)
        for (int y = 0; y < x; y++)
            for (int z = 0; z < y; z++) {
                std::array<uint8_t, 3> best = {255, 255, 255};
                for (auto& p : perms) {
                    std::array<uint8_t, 3> t = {permute_card((Card)x, p), permute_card((Card)y, p),
                                                permute_card((Card)z, p)};
                    std::sort(t.begin(), t.end(), [](uint8_t a, uint8_t b) { return a > b; });
                    if (t < best) best = t;
                }
                classes[best] += 1;
            }
    std::vector<std::pair<std::string, uint32_t>> out;
    for (auto it = classes.rbegin(); it != classes.rend(); ++it)
        out.push_back({card_str(it->first[0]) + card_str(it->first[1]) + card_str(it->first[2]), it->second});
    return out;
}
static std::vector<std::pair<std::string, uint32_t>> canonical_flops_subset(size_t n) {
    auto all = canonical_flops();
    if (n == 0 || n >= all.size()) return all;
    double total = 0;
    for (auto& x : all) total += (double)x.second;
    std::vector<std::pair<std::string, uint32_t>> out;
    double cum = 0;
    size_t ti = 0;
    for (auto& x : all) {
        cum += (double)x.second;
        uint32_t mult = 0;
        while (ti < n && (((double)ti + 0.5) / (double)n) * total <= cum) { mult++; ti++; }
        if (mult > 0) out.push_back({x.first, mult});
    }
    return out;
}

// ------------------------------------------------------------ evaluator.rs
static inline uint32_t make_value(uint32_t cat, const uint8_t* ranks, int n) {  // evaluator.rs:22-28
    uint32_t v = cat;
    for (int slot = 0; slot < 5; slot++) v = (v << 4) | (slot < n ? ranks[slot] : 0u);
    return v;
}
static int straight_top(uint16_t rank_mask) {  // evaluator.rs:33-49
    uint32_t m = ((uint32_t)rank_mask << 1) | (((uint32_t)rank_mask >> 12) & 1u);
    uint32_t run = 0;
    int best = -1;
    for (int i = 0; i < 14; i++) {
        if (m & (1u << i)) {
            run++;
            if (run >= 5) best = i - 1;
        } else {
            run = 0;
        }
    }
    return best;
}
static int top_ranks(uint16_t mask, int n, uint8_t* out) {  // evaluator.rs:53-65
    int count = 0;
    for (int r = 12; r >= 0; r--)
        if (mask & (1u << r)) {
            out[count++] = (uint8_t)r;
            if (count == n) break;
        }
    return count;
}
static uint32_t evaluate7(const Card* cards) {  // evaluator.rs:68-175
    uint16_t suit_masks[4] = {0, 0, 0, 0};
    uint8_t rank_counts[13] = {0};
    uint16_t rank_mask = 0;
    for (int k = 0; k < 7; k++) {
        int r = cards[k] >> 2;
        suit_masks[cards[k] & 3] |= (uint16_t)(1u << r);
        rank_counts[r]++;
        rank_mask |= (uint16_t)(1u << r);
    }
    int flush_suit = -1;
    for (int s = 0; s < 4; s++)
        if (__builtin_popcount(suit_masks[s]) >= 5) { flush_suit = s; break; }
    if (flush_suit >= 0) {
        int top = straight_top(suit_masks[flush_suit]);
        if (top >= 0) { uint8_t r[1] = {(uint8_t)top}; return make_value(8, r, 1); }
    }
    int quads = -1, n_trips = 0, n_pairs = 0;
    uint8_t trips[2] = {0, 0}, pairs[3] = {0, 0, 0};
    for (int r = 12; r >= 0; r--) {
        switch (rank_counts[r]) {
            case 4: quads = r; break;
            case 3: if (n_trips < 2) trips[n_trips++] = (uint8_t)r; break;
            case 2: if (n_pairs < 3) pairs[n_pairs++] = (uint8_t)r; break;
            default: break;
        }
    }
    if (quads >= 0) {
        uint8_t kick[5] = {0};
        top_ranks((uint16_t)(rank_mask & ~(1u << quads)), 1, kick);
        uint8_t r[2] = {(uint8_t)quads, kick[0]};
        return make_value(7, r, 2);
    }
    if (n_trips >= 1) {
        int pr = n_trips >= 2 ? trips[1] : (n_pairs >= 1 ? pairs[0] : -1);
        if (pr >= 0) { uint8_t r[2] = {trips[0], (uint8_t)pr}; return make_value(6, r, 2); }
    }
    if (flush_suit >= 0) {
        uint8_t tops[5] = {0};
        top_ranks(suit_masks[flush_suit], 5, tops);
        return make_value(5, tops, 5);
    }
    int st = straight_top(rank_mask);
    if (st >= 0) { uint8_t r[1] = {(uint8_t)st}; return make_value(4, r, 1); }
    if (n_trips >= 1) {
        uint8_t kick[5] = {0};
        top_ranks((uint16_t)(rank_mask & ~(1u << trips[0])), 2, kick);
        uint8_t r[3] = {trips[0], kick[0], kick[1]};
        return make_value(3, r, 3);
    }
    if (n_pairs >= 2) {
        uint8_t kick[5] = {0};
        top_ranks((uint16_t)(rank_mask & ~(1u << pairs[0]) & ~(1u << pairs[1])), 1, kick);
        uint8_t r[3] = {pairs[0], pairs[1], kick[0]};
        return make_value(2, r, 3);
    }
    if (n_pairs == 1) {
        uint8_t kick[5] = {0};
        top_ranks((uint16_t)(rank_mask & ~(1u << pairs[0])), 3, kick);
        uint8_t r[4] = {pairs[0], kick[0], kick[1], kick[2]};
        return make_value(1, r, 4);
    }
    uint8_t tops[5] = {0};
    top_ranks(rank_mask, 5, tops);
    return make_value(0, tops, 5);
}

// Independent best-of-21 five-card evaluator, restating the reference's own
// test oracle (evaluator.rs:209-290).
struct RefVal {
    uint32_t cat;
    std::vector<uint8_t> r;
    bool operator<(const RefVal& o) const {
        if (cat != o.cat) return cat < o.cat;
        return std::lexicographical_compare(r.begin(), r.end(), o.r.begin(), o.r.end());
    }
};
static RefVal ref_eval5(const Card* c) {
    std::vector<uint8_t> ranks(5);
    for (int i = 0; i < 5; i++) ranks[i] = c[i] >> 2;
    std::sort(ranks.begin(), ranks.end(), std::greater<uint8_t>());
    bool flush = true;
    for (int i = 1; i < 5; i++) flush &= (c[i] & 3) == (c[0] & 3);
    std::map<uint8_t, uint8_t> counts;
    for (auto r : ranks) counts[r]++;
    std::vector<std::pair<uint8_t, uint8_t>> groups;  // (count, rank)
    for (auto& kv : counts) groups.push_back({kv.second, kv.first});
    std::sort(groups.begin(), groups.end(), std::greater<std::pair<uint8_t, uint8_t>>());
    std::vector<uint8_t> uniq;
    for (auto& kv : counts) uniq.push_back(kv.first);
    std::sort(uniq.begin(), uniq.end(), std::greater<uint8_t>());
    int sh = -1;
    if (uniq.size() == 5) {
        if (uniq[0] - uniq[4] == 4) sh = uniq[0];
        else if (uniq == std::vector<uint8_t>{12, 3, 2, 1, 0}) sh = 3;
    }
    if (flush) {
        if (sh >= 0) return {8, {(uint8_t)sh}};
        return {5, ranks};
    }
    if (groups[0].first == 4) return {7, {groups[0].second, groups[1].second}};
    if (groups[0].first == 3) {
        if (groups[1].first == 2) return {6, {groups[0].second, groups[1].second}};
        return {3, {groups[0].second, groups[1].second, groups[2].second}};
    }
    if (groups[0].first == 2) {
        if (groups[1].first == 2) return {2, {groups[0].second, groups[1].second, groups[2].second}};
        return {1, {groups[0].second, groups[1].second, groups[2].second, groups[3].second}};
    }
    if (sh >= 0) return {4, {(uint8_t)sh}};
    return {0, ranks};
}
static RefVal ref_eval7(const Card* c) {
    bool have = false;
    RefVal best;
    for (int i = 0; i < 7; i++)
        for (int j = i + 1; j < 7; j++) {
            Card f[5];
            int n = 0;
            for (int k = 0; k < 7; k++) if (k != i && k != j) f[n++] = c[k];
            RefVal v = ref_eval5(f);
            if (!have || best < v) { best = v; have = true; }
        }
    return best;
}

// ---------------------------------------------------------------- range.rs
enum Suited { PAIR, SUITED, OFFSUIT };
static std::vector<std::pair<Card, Card>> class_combo_list(int hi, int lo, Suited s) {  // range.rs:141-176
    std::vector<std::pair<Card, Card>> out;
    if (s == PAIR) {
        if (hi != lo) return out;
        for (int s1 = 0; s1 < 4; s1++)
            for (int s2 = 0; s2 < s1; s2++) out.push_back({make_card(hi, s1), make_card(lo, s2)});
    } else if (s == SUITED) {
        if (hi == lo) return out;
        for (int su = 0; su < 4; su++) out.push_back({make_card(hi, su), make_card(lo, su)});
    } else {
        if (hi == lo) return out;
        for (int s1 = 0; s1 < 4; s1++)
            for (int s2 = 0; s2 < 4; s2++)
                if (s1 != s2) out.push_back({make_card(hi, s1), make_card(lo, s2)});
    }
    return out;
}
static std::vector<std::pair<Card, Card>> expand_class(int hi, int lo, char marker) {  // range.rs:178-200
    std::vector<std::pair<Card, Card>> out;
    if (hi == lo) {
        if (marker) fail("pairs cannot have a suitedness marker");
        return class_combo_list(hi, lo, PAIR);
    }
    if (marker == 's') return class_combo_list(hi, lo, SUITED);
    if (marker == 'o') return class_combo_list(hi, lo, OFFSUIT);
    if (marker == 0) {
        out = class_combo_list(hi, lo, SUITED);
        auto o = class_combo_list(hi, lo, OFFSUIT);
        out.insert(out.end(), o.begin(), o.end());
        return out;
    }
    fail("invalid suitedness marker");
}
static bool parse_class(const std::string& s, int* hi, int* lo, char* marker) {  // range.rs:203-221
    if (s.size() < 2 || s.size() > 3) return false;
    int r1 = rank_from_char(s[0]), r2 = rank_from_char(s[1]);
    if (r1 < 0 || r2 < 0) return false;
    char m = 0;
    if (s.size() == 3) {
        m = (char)tolower((unsigned char)s[2]);
        if (m != 's' && m != 'o') return false;
    }
    *hi = std::max(r1, r2);
    *lo = std::min(r1, r2);
    *marker = m;
    return true;
}
static std::vector<std::pair<Card, Card>> expand_item(const std::string& item0) {  // range.rs:223-303
    std::string item = trim(item0);
    if (item.size() == 4 && rank_from_char(item[0]) >= 0 && suit_from_char(item[1]) >= 0 &&
        rank_from_char(item[2]) >= 0 && suit_from_char(item[3]) >= 0) {
        Card c1 = card_from_str(item.substr(0, 2)), c2 = card_from_str(item.substr(2, 2));
        if (c1 == c2) fail("combo with duplicate card: " + item);
        return {{c1, c2}};
    }
    size_t dash = item.find('-');
    if (dash != std::string::npos) {
        int h1, l1, h2, l2;
        char m1, m2;
        if (!parse_class(trim(item.substr(0, dash)), &h1, &l1, &m1)) fail("invalid range start: " + item);
        if (!parse_class(trim(item.substr(dash + 1)), &h2, &l2, &m2)) fail("invalid range end: " + item);
        if (m1 != m2) fail("mismatched suitedness in range: " + item);
        std::vector<std::pair<Card, Card>> out;
        auto add = [&](const std::vector<std::pair<Card, Card>>& v) { out.insert(out.end(), v.begin(), v.end()); };
        if (h1 == l1 && h2 == l2) {
            int top = std::max(h1, h2), bot = std::min(h1, h2);
            for (int r = bot; r <= top; r++) add(expand_class(r, r, m1));
        } else if (h1 == h2) {
            int top = std::max(l1, l2), bot = std::min(l1, l2);
            for (int r = bot; r <= top; r++) {
                if (r == h1) continue;
                add(expand_class(h1, r, m1));
            }
        } else if (h1 - l1 == h2 - l2) {
            int top = std::max(h1, h2), bot = std::min(h1, h2), gap = h1 - l1;
            for (int h = bot; h <= top; h++) add(expand_class(h, h - gap, m1));
        } else {
            fail("unsupported range shape: " + item);
        }
        return out;
    }
    if (!item.empty() && item.back() == '+') {
        int hi, lo;
        char m;
        if (!parse_class(trim(item.substr(0, item.size() - 1)), &hi, &lo, &m)) fail("invalid item: " + item);
        std::vector<std::pair<Card, Card>> out;
        if (hi == lo) {
            for (int r = hi; r < 13; r++) { auto v = expand_class(r, r, m); out.insert(out.end(), v.begin(), v.end()); }
        } else {
            for (int l = lo; l < hi; l++) { auto v = expand_class(hi, l, m); out.insert(out.end(), v.begin(), v.end()); }
        }
        return out;
    }
    int hi, lo;
    char m;
    if (!parse_class(item, &hi, &lo, &m)) fail("invalid range token: " + item);
    return expand_class(hi, lo, m);
}
static std::vector<float> parse_range(const std::string& s) {  // range.rs:28-58
    std::vector<float> w(1326, 0.0f);
    std::string norm = s;
    for (char& c : norm) if (c == '\n' || c == '\t' || c == ';') c = ',';
    size_t i = 0;
    while (i <= norm.size()) {
        size_t j = i;
        while (j < norm.size() && norm[j] != ',' && norm[j] != ' ') j++;
        std::string token = trim(norm.substr(i, j - i));
        i = j + 1;
        if (token.empty()) continue;
        std::string item = token;
        float weight = 1.0f;
        size_t colon = token.rfind(':');
        if (colon != std::string::npos) {
            item = trim(token.substr(0, colon));
            std::string ws = trim(token.substr(colon + 1));
            char* end = nullptr;
            errno = 0;
            weight = ws.empty() ? NAN : strtof(ws.c_str(), &end);
            if (ws.empty() || *end != 0) fail("invalid weight in token " + token);
            if (weight > 1.0f) weight /= 100.0f;
            if (!(weight >= 0.0f && weight <= 1.0f)) fail("weight out of range in token " + token);
        }
        for (auto& pr : expand_item(item)) w[combo_index(pr.first, pr.second)] = weight;
    }
    return w;
}

// ----------------------------------------------------------------- tree.rs
enum { K_ACTION = 0, K_CHANCE = 1, K_FOLD = 2, K_SHOWDOWN = 3 };
enum { A_FOLD = 0, A_CHECK = 1, A_CALL = 2, A_BET = 3, A_RAISE = 4 };
struct Size { int kind; double v; };  // 0 PotPct 1 PrevMult 2 AllIn (tree.rs:14-21)
struct Sizing { std::vector<Size> bet, raise, donk; };
struct TreeConfig {  // tree.rs:70-95
    double starting_pot = 60, effective_stack = 970, rake_pct = 0, rake_cap = 0, allin_threshold = 0.85;
    bool add_allin = false;
    int max_raises = 10;
    Sizing oop[3], ip[3];
};
struct Action { int kind; double amount; };
struct Node {  // tree.rs:178-198
    uint8_t kind, player, street, num_children;
    uint32_t children_start, actions_start;
    uint64_t data_offset;
    double put[2];
    double t_win, t_lose, t_tie;
};
struct Tree {
    int root_street;
    std::vector<Node> nodes;
    std::vector<uint32_t> children;
    std::vector<Action> actions;
    uint64_t data_size[2] = {0, 0};
};
struct BuildState {  // tree.rs:213-224
    int street, to_act;
    double put[2], street_bet[2], last_increment;
    int num_raises;
    int last_aggressor;  // -1 = None
    bool checked;
};
static void dedupe_amounts(std::vector<double>& v) {  // tree.rs:781-787
    std::stable_sort(v.begin(), v.end(), [](double a, double b) { return a < b; });
    std::vector<double> out;
    for (double x : v) {
        if (!out.empty() && std::fabs(x - out.back()) < 1e-6) continue;
        out.push_back(x);
    }
    v.swap(out);
}
struct TreeBuilder {
    const TreeConfig& cfg;
    int root_street;
    uint64_t board_mask;
    uint64_t max_nodes;  // 0 = none
    uint64_t num_hands[2];
    Tree t;
    TreeBuilder(const TreeConfig& c, int rs, uint64_t bm, uint64_t mx, uint64_t nh0, uint64_t nh1)
        : cfg(c), root_street(rs), board_mask(bm), max_nodes(mx) {
        num_hands[0] = nh0;
        num_hands[1] = nh1;
        t.root_street = rs;
    }
    void check_budget() {  // tree.rs:412-420
        if (max_nodes && t.nodes.size() >= max_nodes)
            fail("tree too large: over the max_nodes budget of " + std::to_string(max_nodes) +
                 "; reduce bet/raise sizes, max_raises, or effective stack");
    }
    const Sizing& sizing(int player, int street) const { return player == 0 ? cfg.oop[street] : cfg.ip[street]; }
    double rake(double pot) const {  // tree.rs:526-533
        double r = cfg.rake_pct * pot;
        return cfg.rake_cap > 0.0 ? std::min(r, cfg.rake_cap) : r;
    }
    std::vector<Action> legal_actions(const BuildState& st) const {  // tree.rs:432-524
        int me = st.to_act, opp = 1 - me;
        double stack_me = cfg.effective_stack - (st.put[me] - cfg.starting_pot / 2.0);
        std::vector<Action> acts;
        double facing = st.street_bet[opp] - st.street_bet[me];
        if (facing > 1e-9) {
            acts.push_back({A_FOLD, 0});
            acts.push_back({A_CALL, st.street_bet[opp]});
            bool can_raise = stack_me > facing + 1e-9 && st.num_raises < cfg.max_raises;
            if (can_raise) {
                double pot_after_call = st.put[0] + st.put[1] + facing;
                double max_to = st.street_bet[me] + stack_me;
                std::vector<double> cand;
                for (const Size& s : sizing(st.to_act, st.street).raise) {
                    double to = s.kind == 0 ? st.street_bet[opp] + s.v / 100.0 * pot_after_call
                              : s.kind == 1 ? st.street_bet[opp] * s.v : max_to;
                    cand.push_back(to);
                }
                if (cfg.add_allin) cand.push_back(max_to);
                double min_to = st.street_bet[opp] + std::max(st.last_increment, 1e-9);
                std::vector<double> tos;
                for (double to : cand) {
                    if (to < min_to) to = min_to;
                    if (to >= max_to - 1e-9 || to >= cfg.allin_threshold * max_to - 1e-9) to = max_to;
                    if (to > st.street_bet[opp] + 1e-9) tos.push_back(to);
                }
                dedupe_amounts(tos);
                for (double to : tos) acts.push_back({A_RAISE, to});
            }
        } else {
            acts.push_back({A_CHECK, 0});
            if (stack_me > 1e-9) {
                const Sizing& sz = sizing(st.to_act, st.street);
                bool donking = st.to_act == 0 && st.street > root_street && st.last_aggressor == 1;
                const std::vector<Size>& list = donking ? sz.donk : sz.bet;
                double pot = st.put[0] + st.put[1];
                double max_to = stack_me;
                std::vector<double> cand;
                for (const Size& s : list) {
                    if (s.kind == 1) continue;
                    cand.push_back(s.kind == 0 ? s.v / 100.0 * pot : max_to);
                }
                if (cfg.add_allin && (!list.empty() || !donking)) cand.push_back(max_to);
                std::vector<double> tos;
                for (double to : cand) {
                    if (to <= 1e-9) continue;
                    if (to >= max_to - 1e-9 || to >= cfg.allin_threshold * max_to - 1e-9) to = max_to;
                    tos.push_back(to);
                }
                dedupe_amounts(tos);
                for (double to : tos) acts.push_back({A_BET, to});
            }
        }
        return acts;
    }
    uint32_t push_node(const Node& n) {
        t.nodes.push_back(n);
        return (uint32_t)(t.nodes.size() - 1);
    }
    static Node blank(int kind, int player, int street, const double* put) {
        Node n;
        n.kind = (uint8_t)kind;
        n.player = (uint8_t)player;
        n.street = (uint8_t)street;
        n.num_children = 0;
        n.children_start = 0;
        n.actions_start = 0;
        n.data_offset = 0;
        n.put[0] = put[0];
        n.put[1] = put[1];
        n.t_win = n.t_lose = n.t_tie = 0.0;
        return n;
    }
    uint32_t action_node(const BuildState& st) {  // tree.rs:535-574
        check_budget();
        std::vector<Action> acts = legal_actions(st);
        size_t n = acts.size();
        if (n == 0 || n > 250) fail("invalid action count during tree build");
        uint32_t astart = (uint32_t)t.actions.size();
        t.actions.insert(t.actions.end(), acts.begin(), acts.end());
        int me = st.to_act;
        uint64_t doff = t.data_size[me];
        t.data_size[me] += (uint64_t)n * num_hands[me];
        Node nd = blank(K_ACTION, st.to_act, st.street, st.put);
        nd.num_children = (uint8_t)n;
        nd.actions_start = astart;
        nd.data_offset = doff;
        uint32_t idx = push_node(nd);
        std::vector<uint32_t> kids;
        for (const Action& a : acts) kids.push_back(apply_action(st, a));
        t.nodes[idx].children_start = (uint32_t)t.children.size();
        t.children.insert(t.children.end(), kids.begin(), kids.end());
        return idx;
    }
    uint32_t apply_action(const BuildState& st, const Action& a) {  // tree.rs:576-652
        int me = st.to_act, opp = 1 - me;
        if (a.kind == A_FOLD) {
            double f = st.put[me];
            double rk = rake(2.0 * f);
            Node nd = blank(K_FOLD, st.to_act, st.street, st.put);
            nd.t_win = f - rk;
            nd.t_lose = -f;
            nd.t_tie = 0.0;
            return push_node(nd);
        }
        if (a.kind == A_CHECK) {
            if (st.checked) return street_end(st.street, st.put, st.last_aggressor, false);
            BuildState ns = st;
            ns.to_act = st.to_act ^ 1;
            ns.checked = true;
            return action_node(ns);
        }
        if (a.kind == A_CALL) {
            double put[2] = {st.put[0], st.put[1]};
            put[me] += a.amount - st.street_bet[me];
            double sa = cfg.effective_stack - (put[me] - cfg.starting_pot / 2.0);
            double osa = cfg.effective_stack - (put[opp] - cfg.starting_pot / 2.0);
            bool allin = sa <= 1e-9 || osa <= 1e-9;
            return street_end(st.street, put, st.to_act ^ 1, allin);
        }
        BuildState ns = st;
        ns.put[me] += a.amount - st.street_bet[me];
        ns.street_bet[me] = a.amount;
        double inc = a.amount - std::max(st.street_bet[opp], st.street_bet[me]);
        ns.to_act = st.to_act ^ 1;
        ns.last_increment = std::max(inc, st.last_increment);
        ns.num_raises = st.num_raises + (a.kind == A_RAISE ? 1 : 0);
        return action_node(ns);
    }
    uint32_t street_end(int street, const double* put, int aggressor, bool allin) {  // tree.rs:662-723
        if (street == 2) return showdown_node(put);
        if (allin) return runout_chance(street, put);
        check_budget();
        int next = street + 1;
        uint32_t idx = push_node(blank(K_CHANCE, 0, next, put));
        std::vector<uint32_t> kids(52, SENTINEL);
        for (int c = 0; c < 52; c++) {
            if (board_mask & (1ull << c)) continue;
            BuildState cs;
            cs.street = next;
            cs.to_act = 0;
            cs.put[0] = put[0];
            cs.put[1] = put[1];
            cs.street_bet[0] = cs.street_bet[1] = 0.0;
            cs.last_increment = 0.0;
            cs.num_raises = 0;
            cs.last_aggressor = aggressor;
            cs.checked = false;
            kids[c] = action_node(cs);
        }
        t.nodes[idx].children_start = (uint32_t)t.children.size();
        t.children.insert(t.children.end(), kids.begin(), kids.end());
        t.nodes[idx].num_children = 52;
        return idx;
    }
    uint32_t runout_chance(int street, const double* put) {  // tree.rs:725-759
        check_budget();
        int next = street + 1;
        uint32_t idx = push_node(blank(K_CHANCE, 0, next, put));
        std::vector<uint32_t> kids(52, SENTINEL);
        for (int c = 0; c < 52; c++) {
            if (board_mask & (1ull << c)) continue;
            kids[c] = next == 2 ? showdown_node(put) : runout_chance(next, put);
        }
        t.nodes[idx].children_start = (uint32_t)t.children.size();
        t.children.insert(t.children.end(), kids.begin(), kids.end());
        t.nodes[idx].num_children = 52;
        return idx;
    }
    uint32_t showdown_node(const double* put) {  // tree.rs:761-778
        double pot = put[0] + put[1];
        double rk = rake(pot);
        Node nd = blank(K_SHOWDOWN, 0, 2, put);
        nd.t_win = put[0] - rk;
        nd.t_lose = -put[0];
        nd.t_tie = -rk / 2.0;
        return push_node(nd);
    }
};
static Tree build_tree(const TreeConfig& cfg, const std::vector<Card>& board, uint64_t nh0, uint64_t nh1,
                       uint64_t max_nodes, bool lenient) {  // tree.rs:287-402
    if (board.size() < 3 || board.size() > 5) fail("board must have 3 to 5 cards");
    if (!(cfg.starting_pot > 0.0 && std::isfinite(cfg.starting_pot)) ||
        !(cfg.effective_stack > 0.0 && std::isfinite(cfg.effective_stack)))
        fail("pot and stacks must be positive finite numbers");
    int rs = (int)board.size() - 3;
    static const char* SN[3] = {"flop", "turn", "river"};
    for (int pl = 0; pl < 2; pl++)
        for (int s = 0; s < 3; s++) {
            const Sizing& z = pl == 0 ? cfg.oop[s] : cfg.ip[s];
            for (const auto* l : {&z.bet, &z.raise, &z.donk})
                for (const Size& x : *l)
                    if (x.kind != 2 && !std::isfinite(x.v))
                        fail(std::string(SN[s]) + (pl ? " IP" : " OOP") + ": size is not a finite number");
        }
    if (!lenient) {
        for (int pl = 0; pl < 2; pl++)
            for (int s = rs; s < 3; s++) {
                const Sizing& z = pl == 0 ? cfg.oop[s] : cfg.ip[s];
                bool donk_used = pl == 0 && s > rs;
                for (const Size& x : z.bet)
                    if (x.kind == 1) fail(std::string(SN[s]) + " bet: raise-only size");
                if (donk_used)
                    for (const Size& x : z.donk)
                        if (x.kind == 1) fail(std::string(SN[s]) + " donk: raise-only size");
            }
    }
    uint64_t bm = 0;
    for (Card c : board) bm |= cmask(c);
    TreeBuilder b(cfg, rs, bm, max_nodes, nh0, nh1);
    double half = cfg.starting_pot / 2.0;
    BuildState st;
    st.street = rs;
    st.to_act = 0;
    st.put[0] = st.put[1] = half;
    st.street_bet[0] = st.street_bet[1] = 0.0;
    st.last_increment = 0.0;
    st.num_raises = 0;
    st.last_aggressor = -1;
    st.checked = false;
    b.action_node(st);
    return std::move(b.t);
}

// ----------------------------------------------------------------- game.rs
struct Hand { Card c1, c2; float weight; uint64_t mask; };
struct RiverEval { std::vector<std::pair<uint32_t, uint16_t>> sorted[2]; };
struct Dealt {
    Card cards[2] = {0, 0};
    int len = 0;
    Dealt push(Card c) const { Dealt d = *this; d.cards[d.len++] = c; return d; }
    bool contains(Card c) const { for (int i = 0; i < len; i++) if (cards[i] == c) return true; return false; }
};
struct Spot {
    std::vector<Card> board;
    uint64_t board_mask = 0;
    TreeConfig cfg;
    Tree tree;
    std::vector<Hand> hands[2];
    std::vector<float> weights[2];
    std::vector<uint32_t> same_combo[2];
    int root_street = 0;
    std::vector<std::unique_ptr<RiverEval>> river;  // keyed as RiverTable::key (game.rs:44-57)
    std::vector<std::array<uint8_t, 4>> suit_perms;
    std::vector<std::vector<uint16_t>> hand_perm[2];

    size_t river_key(const Dealt& d) const {
        if (root_street == 2) return 0;
        if (root_street == 1) return d.cards[0];
        Card a = std::min(d.cards[0], d.cards[1]), b = std::max(d.cards[0], d.cards[1]);
        return (size_t)a * 52 + b;
    }
    const RiverEval& river_get(const Dealt& d) const {
        const auto& e = river.at(river_key(d));
        if (!e) fail("river eval missing");
        return *e;
    }
    std::vector<int> perms_fixing(const Dealt& d) const {  // game.rs:335-344
        std::vector<int> out;
        for (size_t k = 0; k < suit_perms.size(); k++) {
            bool ok = true;
            for (int i = 0; i < d.len; i++) ok &= permute_card(d.cards[i], suit_perms[k]) == d.cards[i];
            if (ok) out.push_back((int)k);
        }
        return out;
    }
};
static std::unique_ptr<RiverEval> eval_board(const Spot& sp, const std::vector<Card>& extra) {  // game.rs:387-413
    auto e = std::make_unique<RiverEval>();
    Card c7[7];
    for (size_t i = 0; i < sp.board.size(); i++) c7[i] = sp.board[i];
    uint64_t em = 0;
    for (size_t i = 0; i < extra.size(); i++) { c7[sp.board.size() + i] = extra[i]; em |= cmask(extra[i]); }
    for (int p = 0; p < 2; p++) {
        auto& v = e->sorted[p];
        for (size_t i = 0; i < sp.hands[p].size(); i++) {
            const Hand& h = sp.hands[p][i];
            if (h.mask & em) continue;
            c7[5] = h.c1;
            c7[6] = h.c2;
            v.push_back({evaluate7(c7), (uint16_t)i});
        }
        std::sort(v.begin(), v.end());
    }
    return e;
}
static void build_river_table(Spot& sp) {  // game.rs:384-462
    int rs = sp.root_street;
    if (rs == 2) {
        sp.river.resize(1);
        sp.river[0] = eval_board(sp, {});
    } else if (rs == 1) {
        sp.river.resize(52);
        for (int c = 0; c < 52; c++)
            if (!(sp.board_mask & cmask((Card)c))) sp.river[c] = eval_board(sp, {(Card)c});
    } else {
        sp.river.resize(52 * 52);
        std::vector<std::pair<int, int>> pairs;
        for (int a = 0; a < 52; a++) {
            if (sp.board_mask & cmask((Card)a)) continue;
            for (int b = a + 1; b < 52; b++)
                if (!(sp.board_mask & cmask((Card)b))) pairs.push_back({a, b});
        }
#pragma omp parallel for schedule(dynamic, 8)
        for (long k = 0; k < (long)pairs.size(); k++) {
            int a = pairs[k].first, b = pairs[k].second;
            sp.river[a * 52 + b] = eval_board(sp, {(Card)a, (Card)b});
        }
    }
}
static Spot* new_spot(const TreeConfig& cfg, const std::string& board_s, const std::string& r0,
                      const std::string& r1, uint64_t max_nodes, bool lenient) {  // game.rs:135-331
    if (cfg.rake_pct >= 1.0) fail("rake_pct is a FRACTION of the pot (0.05 = 5%)");
    if (cfg.rake_pct < 0.0) fail("rake_pct must be >= 0");
    if (cfg.rake_cap < 0.0) fail("rake_cap must be >= 0");
    std::unique_ptr<Spot> sp(new Spot());
    sp->cfg = cfg;
    sp->board = parse_cards(board_s);
    if (sp->board.size() < 3 || sp->board.size() > 5) fail("board must have 3 to 5 cards");
    for (Card c : sp->board) sp->board_mask |= cmask(c);
    sp->root_street = (int)sp->board.size() - 3;
    std::vector<float> ranges[2] = {parse_range(r0), parse_range(r1)};
    for (int p = 0; p < 2; p++) {
        for (int idx = 0; idx < 1326; idx++) {
            float w = ranges[p][idx];
            if (w <= 0.0f) continue;
            Card hi, lo;
            combo_from_index(idx, &hi, &lo);
            uint64_t m = cmask(hi) | cmask(lo);
            if (m & sp->board_mask) continue;
            sp->hands[p].push_back({hi, lo, w, m});
        }
        if (sp->hands[p].empty())
            fail(std::string(p == 0 ? "OOP" : "IP") + " range has no combos left after board card removal");
        if (sp->hands[p].size() > 65535) fail("range too large");
    }
    double pair_mass = 0;
    for (auto& a : sp->hands[0])
        for (auto& b : sp->hands[1])
            if (!(a.mask & b.mask)) pair_mass += (double)a.weight * (double)b.weight;
    if (pair_mass <= 0.0) fail("OOP and IP ranges are mutually impossible");
    for (int p = 0; p < 2; p++) {
        std::unordered_map<int, uint32_t> m;
        const auto& opp = sp->hands[1 - p];
        for (size_t j = 0; j < opp.size(); j++) m[combo_index(opp[j].c1, opp[j].c2)] = (uint32_t)j;
        for (auto& h : sp->hands[p]) {
            auto it = m.find(combo_index(h.c1, h.c2));
            sp->same_combo[p].push_back(it == m.end() ? SENTINEL : it->second);
        }
        for (auto& h : sp->hands[p]) sp->weights[p].push_back(h.weight);
    }
    sp->tree = build_tree(cfg, sp->board, sp->hands[0].size(), sp->hands[1].size(), max_nodes, lenient);
    build_river_table(*sp);
    std::unordered_map<int, uint16_t> idx_of[2];
    for (int p = 0; p < 2; p++)
        for (size_t i = 0; i < sp->hands[p].size(); i++)
            idx_of[p][combo_index(sp->hands[p][i].c1, sp->hands[p][i].c2)] = (uint16_t)i;
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++)
            for (int c = 0; c < 4; c++)
                for (int d = 0; d < 4; d++) {
                    std::array<uint8_t, 4> pm = {(uint8_t)a, (uint8_t)b, (uint8_t)c, (uint8_t)d};
                    bool seen[4] = {false, false, false, false}, okp = true;
                    for (int s : pm) { if (seen[s]) okp = false; seen[s] = true; }
                    if (!okp) continue;
                    bool ok = true;
                    for (Card x : sp->board) ok &= permute_card(x, pm) == x;
                    if (!ok) continue;
                    std::vector<uint16_t> tbl[2];
                    for (int p = 0; p < 2 && ok; p++)
                        for (auto& h : sp->hands[p]) {
                            int pc = combo_index(permute_card(h.c1, pm), permute_card(h.c2, pm));
                            auto it = idx_of[p].find(pc);
                            if (it == idx_of[p].end() ||
                                !(std::fabs(sp->hands[p][it->second].weight - h.weight) < 1e-6f)) { ok = false; break; }
                            tbl[p].push_back(it->second);
                        }
                    if (!ok) continue;
                    sp->suit_perms.push_back(pm);
                    sp->hand_perm[0].push_back(tbl[0]);
                    sp->hand_perm[1].push_back(tbl[1]);
                }
    for (size_t k = 0; k < sp->suit_perms.size(); k++)
        if (sp->suit_perms[k] == std::array<uint8_t, 4>{0, 1, 2, 3}) {
            std::swap(sp->suit_perms[0], sp->suit_perms[k]);
            std::swap(sp->hand_perm[0][0], sp->hand_perm[0][k]);
            std::swap(sp->hand_perm[1][0], sp->hand_perm[1][k]);
            break;
        }
    return sp.release();
}

// Exact terminal sums: the GPU engine's order-independent form of the
// terminal sweeps below.  The reference sums opponent reach in f64 in one
// fixed order (game.rs:478-485, 512-575) and casts each difference to f32.
// Here every reach value r (f32, >= 0) of one opponent vector is put on one
// fixed-point grid -- q = round-half-even(r * 2^S) as an int64, with S = 51 - E
// where the vector's largest value is < 2^E, so q < 2^51 and a sum of at most
// 1326 of them stays below 2^62 -- the sums and differences are exact integer
// arithmetic in any order, and each difference becomes f32 once:
// f32(x) correctly rounded, then scaled by 2^-S.  The grid's step is 2^-51 of
// the vector's top power of two, about the rounding step of the reference's
// f64 running sums; what stays the reference's is everything after the
// casts (same-combo add, tie term, payoff products in f32).
static int fix_scale(float maxv) {
    uint32_t u;
    std::memcpy(&u, &maxv, 4);
    const int e = (int)((u >> 23) & 0xFFu);
    const uint32_t m = u & 0x7FFFFFu;
    if (e == 0 && m == 0) return 0;                                        // all zero
    const int E = e != 0 ? e - 126 : (32 - __builtin_clz(m)) - 149;        // maxv < 2^E
    return 51 - E;
}
static inline float pow2f(int k) {  // 2^k, k in [-126, 127]
    uint32_t u = (uint32_t)(127 + k) << 23;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
static inline int64_t fix_q(float r, int S) {  // round-half-even(r * 2^S); the scalings are exact
    float x = r;
    if (S > 100) { x *= pow2f(100); S -= 100; }
    x *= pow2f(S);
    return (int64_t)std::nearbyint((double)x);  // |x| < 2^52: exact in f64, rounded half-even
}
static inline float fix_f(int64_t v, int S) {  // f32(v * 2^-S): one rounding, then exact scaling
    float y = (float)v;
    if (S > 100) { y *= pow2f(-100); S -= 100; }
    return y * pow2f(-S);
}
static int vec_scale(const float* r, int n) {
    float m = 0.0f;
    for (int j = 0; j < n; j++) m = std::max(m, r[j]);
    return fix_scale(m);
}
static void fold_cfv_exact(const std::vector<Hand>& me, const std::vector<Hand>& opp, const float* reach_o,
                           const std::vector<uint32_t>& same, float amount, float* out) {
    const int S = vec_scale(reach_o, (int)opp.size());
    int64_t t = 0, s[52] = {0};
    for (size_t j = 0; j < opp.size(); j++) {
        const int64_t q = fix_q(reach_o[j], S);
        t += q;
        s[opp[j].c1] += q;
        s[opp[j].c2] += q;
    }
    for (size_t i = 0; i < me.size(); i++) {
        float same_r = same[i] != SENTINEL ? reach_o[same[i]] : 0.0f;
        float valid = fix_f(t - s[me[i].c1] - s[me[i].c2], S) + same_r;
        out[i] = amount * valid;
    }
}
static void showdown_cfv_exact(const RiverEval& ev, int p, const std::vector<Hand>& me, const std::vector<Hand>& opp,
                               const float* reach_o, const std::vector<uint32_t>& same, float win, float lose,
                               float tie, float* out) {
    const auto& mine = ev.sorted[p];
    const auto& opps = ev.sorted[1 - p];
    const int S = vec_scale(reach_o, (int)opp.size());  // the whole opponent vector's scale
    int64_t t_all = 0, s_all[52] = {0};
    for (auto& x : opps) {
        const int64_t q = fix_q(reach_o[x.second], S);
        t_all += q;
        s_all[opp[x.second].c1] += q;
        s_all[opp[x.second].c2] += q;
    }
    std::vector<float> lower(mine.size());
    {
        int64_t t = 0, s[52] = {0};
        size_t j = 0;
        for (size_t k = 0; k < mine.size(); k++) {
            while (j < opps.size() && opps[j].first < mine[k].first) {
                const int64_t q = fix_q(reach_o[opps[j].second], S);
                const Hand& h = opp[opps[j].second];
                t += q;
                s[h.c1] += q;
                s[h.c2] += q;
                j++;
            }
            const Hand& h = me[mine[k].second];
            lower[k] = fix_f(t - s[h.c1] - s[h.c2], S);
        }
    }
    int64_t t = 0, s[52] = {0};
    size_t j = opps.size();
    for (size_t k = mine.size(); k-- > 0;) {
        uint16_t i = mine[k].second;
        while (j > 0 && opps[j - 1].first > mine[k].first) {
            j--;
            const int64_t q = fix_q(reach_o[opps[j].second], S);
            const Hand& h = opp[opps[j].second];
            t += q;
            s[h.c1] += q;
            s[h.c2] += q;
        }
        const Hand& h = me[i];
        float higher = fix_f(t - s[h.c1] - s[h.c2], S);
        float same_r = same[i] != SENTINEL ? reach_o[same[i]] : 0.0f;
        float valid = fix_f(t_all - s_all[h.c1] - s_all[h.c2], S) + same_r;
        float lo = lower[k];
        float ti = valid - lo - higher;
        out[i] = win * lo + lose * higher + tie * ti;
    }
}

// terminal evaluation (game.rs:470-577)
static void showdown_cfv_f64(const RiverEval& ev, int p, const std::vector<Hand>& me, const std::vector<Hand>& opp,
                             const float* reach_o, const std::vector<uint32_t>& same, float win, float lose, float tie,
                             float* out);
static void fold_cfv_f64(const std::vector<Hand>& me, const std::vector<Hand>& opp, const float* reach_o,
                         const std::vector<uint32_t>& same, float amount, float* out);
// sums: 0 = the reference's f64 running sums, 1 = exact fixed-point sums
static void fold_cfv(const std::vector<Hand>& me, const std::vector<Hand>& opp, const float* reach_o,
                     const std::vector<uint32_t>& same, float amount, float* out, int sums) {
    if (sums) fold_cfv_exact(me, opp, reach_o, same, amount, out);
    else fold_cfv_f64(me, opp, reach_o, same, amount, out);
}
static void showdown_cfv(const RiverEval& ev, int p, const std::vector<Hand>& me, const std::vector<Hand>& opp,
                         const float* reach_o, const std::vector<uint32_t>& same, float win, float lose, float tie,
                         float* out, int sums) {
    if (sums) showdown_cfv_exact(ev, p, me, opp, reach_o, same, win, lose, tie, out);
    else showdown_cfv_f64(ev, p, me, opp, reach_o, same, win, lose, tie, out);
}
static void fold_cfv_f64(const std::vector<Hand>& me, const std::vector<Hand>& opp, const float* reach_o,
                         const std::vector<uint32_t>& same, float amount, float* out) {
    double t = 0, s[52] = {0};
    for (size_t j = 0; j < opp.size(); j++) {
        double r = reach_o[j];
        t += r;
        s[opp[j].c1] += r;
        s[opp[j].c2] += r;
    }
    for (size_t i = 0; i < me.size(); i++) {
        float same_r = same[i] != SENTINEL ? reach_o[same[i]] : 0.0f;
        float valid = (float)(t - s[me[i].c1] - s[me[i].c2]) + same_r;
        out[i] = amount * valid;
    }
}
static void showdown_cfv_f64(const RiverEval& ev, int p, const std::vector<Hand>& me, const std::vector<Hand>& opp,
                             const float* reach_o, const std::vector<uint32_t>& same, float win, float lose, float tie,
                             float* out) {
    const auto& mine = ev.sorted[p];
    const auto& opps = ev.sorted[1 - p];
    double t_all = 0, s_all[52] = {0};
    for (auto& x : opps) {
        double r = reach_o[x.second];
        t_all += r;
        s_all[opp[x.second].c1] += r;
        s_all[opp[x.second].c2] += r;
    }
    std::vector<float> lower(mine.size());
    {
        double t = 0, s[52] = {0};
        size_t j = 0;
        for (size_t k = 0; k < mine.size(); k++) {
            uint32_t st = mine[k].first;
            while (j < opps.size() && opps[j].first < st) {
                double r = reach_o[opps[j].second];
                const Hand& h = opp[opps[j].second];
                t += r;
                s[h.c1] += r;
                s[h.c2] += r;
                j++;
            }
            const Hand& h = me[mine[k].second];
            lower[k] = (float)(t - s[h.c1] - s[h.c2]);
        }
    }
    {
        double t = 0, s[52] = {0};
        size_t j = opps.size();
        for (size_t k = mine.size(); k-- > 0;) {
            uint32_t st = mine[k].first;
            uint16_t i = mine[k].second;
            while (j > 0 && opps[j - 1].first > st) {
                j--;
                double r = reach_o[opps[j].second];
                const Hand& h = opp[opps[j].second];
                t += r;
                s[h.c1] += r;
                s[h.c2] += r;
            }
            const Hand& h = me[i];
            float higher = (float)(t - s[h.c1] - s[h.c2]);
            float same_r = same[i] != SENTINEL ? reach_o[same[i]] : 0.0f;
            float valid = (float)(t_all - s_all[h.c1] - s_all[h.c2]) + same_r;
            float lo = lower[k];
            float ti = valid - lo - higher;
            out[i] = win * lo + lose * higher + tie * ti;
        }
    }
}
// All-double twins used only by the FP64 best-response oracle.
static void fold_cfv64(const std::vector<Hand>& me, const std::vector<Hand>& opp, const double* reach_o,
                       const std::vector<uint32_t>& same, double amount, double* out) {
    double t = 0, s[52] = {0};
    for (size_t j = 0; j < opp.size(); j++) { t += reach_o[j]; s[opp[j].c1] += reach_o[j]; s[opp[j].c2] += reach_o[j]; }
    for (size_t i = 0; i < me.size(); i++) {
        double same_r = same[i] != SENTINEL ? reach_o[same[i]] : 0.0;
        out[i] = amount * (t - s[me[i].c1] - s[me[i].c2] + same_r);
    }
}
static void showdown_cfv64(const RiverEval& ev, int p, const std::vector<Hand>& me, const std::vector<Hand>& opp,
                           const double* reach_o, const std::vector<uint32_t>& same, double win, double lose,
                           double tie, double* out) {
    const auto& mine = ev.sorted[p];
    const auto& opps = ev.sorted[1 - p];
    double t_all = 0, s_all[52] = {0};
    for (auto& x : opps) { double r = reach_o[x.second]; t_all += r; s_all[opp[x.second].c1] += r; s_all[opp[x.second].c2] += r; }
    std::vector<double> lower(mine.size());
    double t = 0, s[52] = {0};
    size_t j = 0;
    for (size_t k = 0; k < mine.size(); k++) {
        while (j < opps.size() && opps[j].first < mine[k].first) {
            double r = reach_o[opps[j].second]; const Hand& h = opp[opps[j].second];
            t += r; s[h.c1] += r; s[h.c2] += r; j++;
        }
        const Hand& h = me[mine[k].second];
        lower[k] = t - s[h.c1] - s[h.c2];
    }
    t = 0;
    std::fill(s, s + 52, 0.0);
    j = opps.size();
    for (size_t k = mine.size(); k-- > 0;) {
        while (j > 0 && opps[j - 1].first > mine[k].first) {
            j--; double r = reach_o[opps[j].second]; const Hand& h = opp[opps[j].second];
            t += r; s[h.c1] += r; s[h.c2] += r;
        }
        uint16_t i = mine[k].second;
        const Hand& h = me[i];
        double higher = t - s[h.c1] - s[h.c2];
        double same_r = same[i] != SENTINEL ? reach_o[same[i]] : 0.0;
        double valid = t_all - s_all[h.c1] - s_all[h.c2] + same_r;
        out[i] = win * lower[k] + lose * higher + tie * (valid - lower[k] - higher);
    }
}

// ---------------------------------------------------------------- store.rs
static inline int16_t sat_i16(float x) {  // Rust `as i16`: saturating, NaN -> 0
    if (std::isnan(x)) return 0;
    if (x >= 32767.0f) return 32767;
    if (x <= -32768.0f) return -32768;
    return (int16_t)x;
}
static inline uint16_t sat_u16(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 65535.0f) return 65535;
    if (x <= 0.0f) return 0;
    return (uint16_t)x;
}
static float quantize_i16(const float* src, int n, float max, int16_t* dst) {  // store.rs:171-181
    if (!(max > 0.0f && std::isfinite(max))) { std::fill(dst, dst + n, (int16_t)0); return 0.0f; }
    float k = 32767.0f / max;
    for (int i = 0; i < n; i++) dst[i] = sat_i16(std::nearbyint(src[i] * k));
    return max;
}
static float quantize_u16(const float* src, int n, float max, uint16_t* dst) {  // store.rs:185-195
    if (!(max > 0.0f && std::isfinite(max))) { std::fill(dst, dst + n, (uint16_t)0); return 0.0f; }
    float k = 65535.0f / max;
    for (int i = 0; i < n; i++) dst[i] = sat_u16(std::nearbyint(std::fmax(src[i], 0.0f) * k));
    return max;
}
// Stochastic rounding of the 16-bit requantisation (the engine's optional
// rounding mode; store.rs rounds to nearest even): x -> floor(x + u) with u in
// [0, 1) from the lowbias32 integer hash (Chris Wellons, "Hash Prospector",
// public domain): base = h(node ^ h(iteration)), bits = h(base + (hand << 4 |
// action) * 0x9E3779B9); the low 16 bits feed the regret, the high 16 the
// strategy sum.
static inline uint32_t lowbias32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
static inline uint32_t sr_bits(uint32_t node, uint32_t t, uint32_t hand, uint32_t action) {
    const uint32_t base = lowbias32(node ^ lowbias32(t));
    return lowbias32(base + ((hand << 4) | action) * 0x9E3779B9u);
}
static inline float sr_u_lo(uint32_t h) { return (float)(h & 0xFFFFu) * 0x1p-16f; }
static inline float sr_u_hi(uint32_t h) { return (float)(h >> 16) * 0x1p-16f; }
static inline int16_t sr_i16(float x, float u) {  // floor(x + u), saturating, NaN -> 0
    float y = x + u;
    if (y != y) return 0;
    y = std::floor(y);
    return (int16_t)std::fmin(32767.0f, std::fmax(-32768.0f, y));
}
static inline uint16_t sr_u16(float x, float u) {
    float y = x + u;
    if (y != y) return 0;
    y = std::floor(y);
    return (uint16_t)std::fmin(65535.0f, std::fmax(0.0f, y));
}
// quantize_i16 / quantize_u16 with stochastic rounding; src and dst are the
// node's action-major block (entry a * h + i), t the iteration.
static float quantize_i16_sr(const float* src, int na, int h, float max, uint32_t node, uint32_t t, int16_t* dst) {
    if (!(max > 0.0f && std::isfinite(max))) { std::fill(dst, dst + na * h, (int16_t)0); return 0.0f; }
    float k = 32767.0f / max;
    for (int a = 0; a < na; a++)
        for (int i = 0; i < h; i++) dst[a * h + i] = sr_i16(src[a * h + i] * k, sr_u_lo(sr_bits(node, t, i, a)));
    return max;
}
static float quantize_u16_sr(const float* src, int na, int h, float max, uint32_t node, uint32_t t, uint16_t* dst) {
    if (!(max > 0.0f && std::isfinite(max))) { std::fill(dst, dst + na * h, (uint16_t)0); return 0.0f; }
    float k = 65535.0f / max;
    for (int a = 0; a < na; a++)
        for (int i = 0; i < h; i++)
            dst[a * h + i] = sr_u16(std::fmax(src[a * h + i], 0.0f) * k, sr_u_hi(sr_bits(node, t, i, a)));
    return max;
}
static float encode_i16(const float* src, int n, int16_t* dst) {  // store.rs:199-205
    float m = 0.0f;
    for (int i = 0; i < n; i++) m = std::fmax(m, std::fabs(src[i]));
    return quantize_i16(src, n, m, dst);
}
static float encode_u16(const float* src, int n, uint16_t* dst) {  // store.rs:209-215
    float m = 0.0f;
    for (int i = 0; i < n; i++) m = std::fmax(m, src[i]);
    return quantize_u16(src, n, m, dst);
}
static void decode_i16(const int16_t* q, int n, float scale, float* out) {  // store.rs:153-158
    float k = scale / 32767.0f;
    for (int i = 0; i < n; i++) out[i] = (float)q[i] * k;
}
static void decode_u16(const uint16_t* q, int n, float scale, float* out) {  // store.rs:161-166
    float k = scale / 65535.0f;
    for (int i = 0; i < n; i++) out[i] = (float)q[i] * k;
}

// ------------------------------------------------ FP8 (E4M3) arenas
// Not in the reference: the 8-bit arena format of the precision study.  OCP
// FP8 E4M3: 1 sign bit, 4 exponent bits (bias 7), 3 mantissa bits, no
// infinities, S.1111.111 is NaN, the largest finite value is 448.  Encoding
// rounds to nearest, ties to even, and saturates to +-448 (the device's cvt
// to e4m3 with satfinite).  A node's block is stored as v * (448 / max|v|)
// with the max kept as the node's scale, like the 16-bit format.
static uint8_t f32_to_e4m3(float x) {
    if (std::isnan(x)) return 0x7F;
    const uint8_t sign = std::signbit(x) ? 0x80 : 0x00;
    const float a = std::fabs(x);
    if (a >= 448.0f) return sign | 0x7E;
    if (a == 0.0f) return sign;
    int e2 = 0;
    std::frexp(a, &e2);
    int E = e2 - 1;  // a in [2^E, 2^(E+1))
    if (E < -6) {    // subnormals: m * 2^-9, m in 0..7; 8 is the smallest normal
        const float m = std::nearbyint(a * 512.0f);
        return m >= 8.0f ? (uint8_t)(sign | 0x08) : (uint8_t)(sign | (uint8_t)m);
    }
    float m = std::nearbyint(std::ldexp(a, 3 - E));  // (8 + M), exact scaling then RNE
    if (m >= 16.0f) { m = 8.0f; E += 1; }
    const int ef = E + 7;
    if (ef > 15 || (ef == 15 && m > 14.0f)) return sign | 0x7E;
    return (uint8_t)(sign | (ef << 3) | (int)(m - 8.0f));
}
static float e4m3_to_f32(uint8_t q) {
    const int E = (q >> 3) & 15, M = q & 7;
    float v;
    if (E == 15 && M == 7) v = NAN;
    else if (E == 0) v = std::ldexp((float)M, -9);
    else v = std::ldexp((float)(8 + M), E - 10);
    return (q & 0x80) ? -v : v;
}
static float quantize_fp8(const float* src, int n, float max, bool nonneg, uint8_t* dst) {
    if (!(max > 0.0f && std::isfinite(max))) { std::fill(dst, dst + n, (uint8_t)0); return 0.0f; }
    float k = 448.0f / max;
    for (int i = 0; i < n; i++) dst[i] = f32_to_e4m3(nonneg ? std::fmax(src[i], 0.0f) * k : src[i] * k);
    return max;
}
static float encode_fp8(const float* src, int n, bool nonneg, uint8_t* dst) {
    float m = 0.0f;
    for (int i = 0; i < n; i++) m = std::fmax(m, nonneg ? src[i] : std::fabs(src[i]));
    return quantize_fp8(src, n, m, nonneg, dst);
}
static void decode_fp8(const uint8_t* q, int n, float scale, float* out) {
    float k = scale / 448.0f;
    for (int i = 0; i < n; i++) out[i] = e4m3_to_f32(q[i]) * k;
}

// One arena (store.rs:79-150): f32, or 16-bit quants with a per-node scale
// (or, for the precision study, FP8 E4M3 with a per-node scale).
struct Store {
    int kind = 0;  // 0 f32, 1 i16, 2 u16, 3 fp8 (signed), 4 fp8 (strategy sums, >= 0)
    std::vector<float> f;
    std::vector<int16_t> qi;
    std::vector<uint16_t> qu;
    std::vector<uint8_t> q8;
    std::vector<float> scale;
    void init(int k, uint64_t len, size_t nodes) {
        kind = k;
        if (k == 0) f.assign(len, 0.0f);
        else if (k == 1) { qi.assign(len, 0); scale.assign(nodes, 0.0f); }
        else if (k == 2) { qu.assign(len, 0); scale.assign(nodes, 0.0f); }
        else { q8.assign(len, 0); scale.assign(nodes, 0.0f); }
    }
    void read_f32(uint32_t node, uint64_t off, int n, float* out) const {
        if (kind == 0) std::memcpy(out, f.data() + off, sizeof(float) * n);
        else if (kind == 1) decode_i16(qi.data() + off, n, scale[node], out);
        else if (kind == 2) decode_u16(qu.data() + off, n, scale[node], out);
        else decode_fp8(q8.data() + off, n, scale[node], out);
    }
    void write_f32(uint32_t node, uint64_t off, int n, const float* src) {
        if (kind == 0) std::memcpy(f.data() + off, src, sizeof(float) * n);
        else if (kind == 1) scale[node] = encode_i16(src, n, qi.data() + off);
        else if (kind == 2) scale[node] = encode_u16(src, n, qu.data() + off);
        else scale[node] = encode_fp8(src, n, kind == 4, q8.data() + off);
    }
};

// ------------------------------------------------------------------ cfr.rs
enum { DCFR = 0, CFRPLUS = 1, PCFRPLUS = 2 };
struct Disc { float pos, neg, strat; };
static Disc discounts(int algo, uint32_t it) {  // cfr.rs:44-64
    double t = (double)it;
    Disc d;
    double q = t / (t + 1.0);
    if (algo == DCFR) {
        double ta = std::pow(t, 1.5);
        d.pos = (float)(ta / (ta + 1.0));
        d.neg = 0.5f;
        d.strat = (float)(q * q);
    } else {
        d.pos = 1.0f;
        d.neg = 0.0f;
        d.strat = (float)(q * q);
    }
    return d;
}
static void regret_match(const float* r, int na, int nh, float* sig) {  // cfr.rs:875-895
    for (int i = 0; i < nh; i++) {
        float sum = 0.0f;
        for (int a = 0; a < na; a++) sum += std::fmax(r[a * nh + i], 0.0f);
        if (sum > 1e-12f) {
            float inv = 1.0f / sum;
            for (int a = 0; a < na; a++) sig[a * nh + i] = std::fmax(r[a * nh + i], 0.0f) * inv;
        } else {
            float u = 1.0f / (float)na;
            for (int a = 0; a < na; a++) sig[a * nh + i] = u;
        }
    }
}
static void regret_match_q(const int16_t* q, int na, int nh, float* sig) {  // cfr.rs:899-919
    for (int i = 0; i < nh; i++) {
        int32_t sum = 0;
        for (int a = 0; a < na; a++) sum += std::max<int32_t>(q[a * nh + i], 0);
        if (sum > 0) {
            float inv = 1.0f / (float)sum;
            for (int a = 0; a < na; a++) sig[a * nh + i] = (float)std::max<int32_t>(q[a * nh + i], 0) * inv;
        } else {
            float u = 1.0f / (float)na;
            for (int a = 0; a < na; a++) sig[a * nh + i] = u;
        }
    }
}
static void regret_match_inplace(float* sig, int na, int nh) {  // cfr.rs:923-942
    for (int i = 0; i < nh; i++) {
        float sum = 0.0f;
        for (int a = 0; a < na; a++) sum += std::fmax(sig[a * nh + i], 0.0f);
        if (sum > 1e-12f) {
            float inv = 1.0f / sum;
            for (int a = 0; a < na; a++) sig[a * nh + i] = std::fmax(sig[a * nh + i], 0.0f) * inv;
        } else {
            float u = 1.0f / (float)na;
            for (int a = 0; a < na; a++) sig[a * nh + i] = u;
        }
    }
}

struct Solver {
    Spot* spot;
    bool compressed;  // 16-bit (mode 1) or FP8 (mode 2) arenas
    int mode;         // 0 f32, 1 i16/u16, 2 fp8
    int algo;
    bool use_iso;
    bool prune;
    int sums = 0;  // terminal sums: 0 = the reference's f64 running sums, 1 = exact fixed point (the GPU's)
    int sr = 0;    // 16-bit requantisation: 0 round to nearest even (store.rs), 1 stochastic rounding
    Store regrets[2], strat[2];
    bool have_preds = false;
    Store preds[2];
    uint32_t iteration = 0;
    std::map<uint32_t, std::vector<float>> locks;
    bool sym_dirty = false;

    Solver(Spot* s, int storage_mode, int al, bool iso, bool pr)
        : spot(s), compressed(storage_mode != 0), mode(storage_mode), algo(al), use_iso(iso), prune(pr) {
        size_t nn = s->tree.nodes.size();
        for (int p = 0; p < 2; p++) {
            regrets[p].init(mode == 0 ? 0 : mode == 1 ? 1 : 3, s->tree.data_size[p], nn);
            strat[p].init(mode == 0 ? 0 : mode == 1 ? 2 : 4, s->tree.data_size[p], nn);
        }
    }
    void ensure_preds() {  // cfr.rs:157-168
        if (have_preds) return;
        size_t nn = spot->tree.nodes.size();
        for (int p = 0; p < 2; p++) preds[p].init(mode == 0 ? 0 : mode == 1 ? 1 : 3, spot->tree.data_size[p], nn);
        have_preds = true;
    }
    int nh(int p) const { return (int)spot->hands[p].size(); }
    const Node& node(uint32_t i) const { return spot->tree.nodes[i]; }
    uint32_t child(const Node& n, int a) const { return spot->tree.children[n.children_start + a]; }

    void iterate() {  // cfr.rs:170-190
        if (algo == PCFRPLUS && !have_preds) ensure_preds();
        sym_dirty = true;
        iteration += 1;
        Disc d = discounts(algo, iteration);
        for (int p = 0; p < 2; p++) {
            std::vector<float> out(nh(p), 0.0f);
            cfr(0, p, spot->weights[p].data(), spot->weights[1 - p].data(), Dealt(), d, out.data());
        }
    }

    void current_strategy(uint32_t idx, const Node& n, float* sig) const {  // cfr.rs:240-292
        auto it = locks.find(idx);
        int p = n.player, na = n.num_children, h = nh(p), cnt = na * h;
        if (it != locks.end()) { std::memcpy(sig, it->second.data(), sizeof(float) * cnt); return; }
        uint64_t off = n.data_offset;
        bool pc = algo == PCFRPLUS && have_preds;
        const Store& R = regrets[p];
        if (R.kind == 0) {
            if (!pc) { regret_match(R.f.data() + off, na, h, sig); return; }
            const float* r = R.f.data() + off;
            const float* pr = preds[p].f.data() + off;
            for (int i = 0; i < cnt; i++) sig[i] = std::fmax(r[i], 0.0f) + pr[i];
            regret_match_inplace(sig, na, h);
        } else if (R.kind == 3) {
            // FP8: regret matching on the stored values before scaling (one
            // scale per node: it cancels), predictions decoded for PCFR+
            const uint8_t* qr = R.q8.data() + off;
            if (!pc) {
                for (int i = 0; i < cnt; i++) sig[i] = e4m3_to_f32(qr[i]);
                regret_match_inplace(sig, na, h);
                return;
            }
            float kr = R.scale[idx] / 448.0f;
            const uint8_t* qp = preds[p].q8.data() + off;
            float kp = preds[p].scale[idx] / 448.0f;
            for (int i = 0; i < cnt; i++) sig[i] = std::fmax(e4m3_to_f32(qr[i]), 0.0f) * kr + e4m3_to_f32(qp[i]) * kp;
            regret_match_inplace(sig, na, h);
        } else {
            if (!pc) { regret_match_q(R.qi.data() + off, na, h, sig); return; }
            const int16_t* qr = R.qi.data() + off;
            float kr = R.scale[idx] / 32767.0f;
            const int16_t* qp = preds[p].qi.data() + off;
            float kp = preds[p].scale[idx] / 32767.0f;
            for (int i = 0; i < cnt; i++) sig[i] = (float)std::max<int16_t>(qr[i], 0) * kr + (float)qp[i] * kp;
            regret_match_inplace(sig, na, h);
        }
    }

    void update_node(uint32_t idx, const Node& n, int p, const float* sig, const float* vals, const float* out,
                     const float* reach_p, const Disc& d) {  // cfr.rs:297-409
        int h = nh(p), na = n.num_children, cnt = na * h;
        uint64_t off = n.data_offset;
        bool pc = algo == PCFRPLUS && have_preds;
        if (!compressed) {
            float* R = regrets[p].f.data() + off;
            float* S = strat[p].f.data() + off;
            for (int a = 0; a < na; a++)
                for (int i = 0; i < h; i++) {
                    int b = a * h + i;
                    float r = R[b];
                    float dd = r > 0.0f ? d.pos : d.neg;
                    R[b] = r * dd + (vals[b] - out[i]);
                    S[b] = S[b] * d.strat + reach_p[i] * sig[b];
                }
            if (pc) {
                float* P = preds[p].f.data() + off;
                for (int a = 0; a < na; a++)
                    for (int i = 0; i < h; i++) P[a * h + i] = vals[a * h + i] - out[i];
            }
            return;
        }
        if (mode == 2) {  // FP8, the same steps as the 16-bit branch below
            uint8_t* rq = regrets[p].q8.data() + off;
            uint8_t* sq = strat[p].q8.data() + off;
            float kr = regrets[p].scale[idx] / 448.0f;
            float kss = strat[p].scale[idx] / 448.0f * d.strat;
            std::vector<float> rb(cnt), sb(cnt);
            float rmax = 0.0f, smax = 0.0f;
            for (int a = 0; a < na; a++) {
                for (int i = 0; i < h; i++) {
                    int b = a * h + i;
                    float dv = e4m3_to_f32(rq[b]);
                    float dd = dv > 0.0f ? d.pos : d.neg;
                    float nr = dv * kr * dd + (vals[b] - out[i]);
                    rb[b] = nr;
                    rmax = std::fmax(rmax, std::fabs(nr));
                }
                for (int i = 0; i < h; i++) {
                    int b = a * h + i;
                    float s = e4m3_to_f32(sq[b]) * kss + reach_p[i] * sig[b];
                    sb[b] = s;
                    smax = std::fmax(smax, s);
                }
            }
            regrets[p].scale[idx] = quantize_fp8(rb.data(), cnt, rmax, false, rq);
            strat[p].scale[idx] = quantize_fp8(sb.data(), cnt, smax, true, sq);
            if (pc) {
                float pmax = 0.0f;
                for (int a = 0; a < na; a++)
                    for (int i = 0; i < h; i++) {
                        float delta = vals[a * h + i] - out[i];
                        rb[a * h + i] = delta;
                        pmax = std::fmax(pmax, std::fabs(delta));
                    }
                preds[p].scale[idx] = quantize_fp8(rb.data(), cnt, pmax, false, preds[p].q8.data() + off);
            }
            return;
        }
        int16_t* rq = regrets[p].qi.data() + off;
        uint16_t* sq = strat[p].qu.data() + off;
        float kr = regrets[p].scale[idx] / 32767.0f;
        float kss = strat[p].scale[idx] / 65535.0f * d.strat;
        std::vector<float> rb(cnt), sb(cnt);
        float rmax = 0.0f, smax = 0.0f;
        for (int a = 0; a < na; a++) {
            for (int i = 0; i < h; i++) {
                int b = a * h + i;
                int16_t qv = rq[b];
                float dd = qv > 0 ? d.pos : d.neg;
                float nr = (float)qv * kr * dd + (vals[b] - out[i]);
                rb[b] = nr;
                rmax = std::fmax(rmax, std::fabs(nr));
            }
            for (int i = 0; i < h; i++) {
                int b = a * h + i;
                float s = (float)sq[b] * kss + reach_p[i] * sig[b];
                sb[b] = s;
                smax = std::fmax(smax, s);
            }
        }
        if (sr) {
            regrets[p].scale[idx] = quantize_i16_sr(rb.data(), na, h, rmax, idx, iteration, rq);
            strat[p].scale[idx] = quantize_u16_sr(sb.data(), na, h, smax, idx, iteration, sq);
        } else {
            regrets[p].scale[idx] = quantize_i16(rb.data(), cnt, rmax, rq);
            strat[p].scale[idx] = quantize_u16(sb.data(), cnt, smax, sq);
        }
        if (pc) {
            float pmax = 0.0f;
            for (int a = 0; a < na; a++)
                for (int i = 0; i < h; i++) {
                    float delta = vals[a * h + i] - out[i];
                    rb[a * h + i] = delta;
                    pmax = std::fmax(pmax, std::fabs(delta));
                }
            preds[p].scale[idx] = quantize_i16(rb.data(), cnt, pmax, preds[p].qi.data() + off);
        }
    }

    template <class F>
    void chance_node(const Node& n, int p, const float* reach_p, const float* reach_o, const Dealt& dealt,
                     float* out, F recurse) {  // cfr.rs:539-664
        const Spot& sp = *spot;
        int h = nh(p), ho = nh(1 - p);
        float divisor = (float)(46 - (int)n.street);
        std::vector<Card> cards;
        for (int c = 0; c < 52; c++)
            if (sp.tree.children[n.children_start + c] != SENTINEL && !dealt.contains((Card)c)) cards.push_back((Card)c);
        Card rep_of[52];
        int perm_of[52];
        for (int c = 0; c < 52; c++) { rep_of[c] = 255; perm_of[c] = 0; }
        if (use_iso && sp.suit_perms.size() > 1) {
            std::vector<int> valid = sp.perms_fixing(dealt);
            for (Card c : cards) {
                Card rep = c;
                int k_rep = 0;
                for (int k : valid) {
                    Card pc = permute_card(c, sp.suit_perms[k]);
                    if (pc < rep) { rep = pc; k_rep = k; }
                }
                rep_of[c] = rep;
                perm_of[c] = k_rep;
            }
        } else {
            for (Card c : cards) rep_of[c] = c;
        }
        std::vector<Card> reps;
        for (Card c : cards) if (rep_of[c] == c) reps.push_back(c);
        bool parallel = !cards.empty() && node(sp.tree.children[n.children_start + cards[0]]).kind == K_ACTION;
        std::vector<std::vector<float>> res(reps.size());
        auto run_child = [&](size_t k) {
            Card c = reps[k];
            uint32_t ch = sp.tree.children[n.children_start + c];
            uint64_t cm = cmask(c);
            std::vector<float> rp(h), ro(ho);
            for (int i = 0; i < h; i++) rp[i] = (sp.hands[p][i].mask & cm) ? 0.0f : reach_p[i];
            for (int j = 0; j < ho; j++) ro[j] = (sp.hands[1 - p][j].mask & cm) ? 0.0f : reach_o[j];
            res[k].assign(h, 0.0f);
            recurse(ch, rp.data(), ro.data(), dealt.push(c), res[k].data());
        };
#ifdef _OPENMP
        if (parallel && !omp_in_parallel() && omp_get_max_threads() > 1) {
#pragma omp parallel for schedule(dynamic, 1)
            for (long k = 0; k < (long)reps.size(); k++) run_child((size_t)k);
        } else
#endif
        {
            (void)parallel;
            for (size_t k = 0; k < reps.size(); k++) run_child(k);
        }
        int by_card[52];
        for (int c = 0; c < 52; c++) by_card[c] = -1;
        for (size_t k = 0; k < reps.size(); k++) by_card[reps[k]] = (int)k;
        for (Card c : cards) {
            const float* co = res[by_card[rep_of[c]]].data();
            uint64_t cm = cmask(c);
            if (c == rep_of[c]) {
                for (int i = 0; i < h; i++) if (!(sp.hands[p][i].mask & cm)) out[i] += co[i];
            } else {
                const auto& tbl = sp.hand_perm[p][perm_of[c]];
                for (int i = 0; i < h; i++) if (!(sp.hands[p][i].mask & cm)) out[i] += co[tbl[i]];
            }
        }
        float inv = 1.0f / divisor;
        for (int i = 0; i < h; i++) out[i] *= inv;
    }

    static bool all_nonpos(const float* r, int n) {
        for (int i = 0; i < n; i++) if (r[i] > 0.0f) return false;
        return true;
    }

    void cfr(uint32_t idx, int p, const float* reach_p, const float* reach_o, const Dealt& dealt, const Disc& d,
             float* out) {  // cfr.rs:414-534
        if (prune && all_nonpos(reach_o, nh(1 - p))) return;
        const Node& n = node(idx);
        const Spot& sp = *spot;
        if (n.kind == K_FOLD) {
            float amount = (float)(n.player == p ? n.t_lose : n.t_win);
            fold_cfv(sp.hands[p], sp.hands[1 - p], reach_o, sp.same_combo[p], amount, out, sums);
        } else if (n.kind == K_SHOWDOWN) {
            showdown_cfv(sp.river_get(dealt), p, sp.hands[p], sp.hands[1 - p], reach_o, sp.same_combo[p],
                         (float)n.t_win, (float)n.t_lose, (float)n.t_tie, out, sums);
        } else if (n.kind == K_CHANCE) {
            chance_node(n, p, reach_p, reach_o, dealt, out,
                        [&](uint32_t c, const float* rp, const float* ro, const Dealt& dd, float* o) {
                            cfr(c, p, rp, ro, dd, d, o);
                        });
        } else {
            int na = n.num_children;
            if (n.player == p) {
                int h = nh(p);
                bool locked = locks.count(idx) > 0;
                std::vector<float> sig(na * h), vals(na * h, 0.0f), rb(h);
                current_strategy(idx, n, sig.data());
                for (int a = 0; a < na; a++) {
                    for (int i = 0; i < h; i++) rb[i] = reach_p[i] * sig[a * h + i];
                    cfr(child(n, a), p, rb.data(), reach_o, dealt, d, vals.data() + a * h);
                }
                for (int a = 0; a < na; a++)
                    for (int i = 0; i < h; i++) out[i] += sig[a * h + i] * vals[a * h + i];
                if (!locked) update_node(idx, n, p, sig.data(), vals.data(), out, reach_p, d);
            } else {
                int o = 1 - p, ho = nh(o), h = nh(p);
                std::vector<float> sig(na * ho), rb(ho), co(h);
                current_strategy(idx, n, sig.data());
                for (int a = 0; a < na; a++) {
                    for (int j = 0; j < ho; j++) rb[j] = reach_o[j] * sig[a * ho + j];
                    std::fill(co.begin(), co.end(), 0.0f);
                    cfr(child(n, a), p, reach_p, rb.data(), dealt, d, co.data());
                    for (int i = 0; i < h; i++) out[i] += co[i];
                }
            }
        }
    }

    void solved_strategy_into(const Node& n, float* sig) const {  // cfr.rs:679-726
        int p = n.player, h = nh(p), na = n.num_children;
        const Store& S = strat[p];
        if (S.kind == 0) {
            const float* s = S.f.data() + n.data_offset;
            for (int i = 0; i < h; i++) {
                double sum = 0;
                for (int a = 0; a < na; a++) sum += (double)std::fmax(s[a * h + i], 0.0f);
                if (sum > 1e-12) {
                    for (int a = 0; a < na; a++) sig[a * h + i] = (float)((double)std::fmax(s[a * h + i], 0.0f) / sum);
                } else {
                    float u = 1.0f / (float)na;
                    for (int a = 0; a < na; a++) sig[a * h + i] = u;
                }
            }
        } else if (S.kind == 4) {  // FP8: the f32 rule on the stored values (the scale cancels)
            const uint8_t* q = S.q8.data() + n.data_offset;
            for (int i = 0; i < h; i++) {
                double sum = 0;
                for (int a = 0; a < na; a++) sum += (double)std::fmax(e4m3_to_f32(q[a * h + i]), 0.0f);
                if (sum > 1e-12) {
                    for (int a = 0; a < na; a++)
                        sig[a * h + i] = (float)((double)std::fmax(e4m3_to_f32(q[a * h + i]), 0.0f) / sum);
                } else {
                    float u = 1.0f / (float)na;
                    for (int a = 0; a < na; a++) sig[a * h + i] = u;
                }
            }
        } else {
            const uint16_t* q = S.qu.data() + n.data_offset;
            for (int i = 0; i < h; i++) {
                uint32_t sum = 0;
                for (int a = 0; a < na; a++) sum += q[a * h + i];
                if (sum > 0) {
                    float inv = 1.0f / (float)sum;
                    for (int a = 0; a < na; a++) sig[a * h + i] = (float)q[a * h + i] * inv;
                } else {
                    float u = 1.0f / (float)na;
                    for (int a = 0; a < na; a++) sig[a * h + i] = u;
                }
            }
        }
    }
    void average_strategy_into(uint32_t idx, const Node& n, float* sig) const {  // cfr.rs:668-674
        auto it = locks.find(idx);
        if (it != locks.end()) { std::memcpy(sig, it->second.data(), sizeof(float) * it->second.size()); return; }
        solved_strategy_into(n, sig);
    }

    // ------------------------------------------------- best_response.rs
    void br_into(uint32_t idx, int p, const float* reach_o, const Dealt& dealt, float* out, bool avg_mode) {
        // best_response.rs:19-124 (avg_mode = false) and 135-223 (avg_mode = true)
        int ho = nh(1 - p), h = nh(p);
        if (all_nonpos(reach_o, ho)) return;
        const Node& n = node(idx);
        const Spot& sp = *spot;
        if (n.kind == K_FOLD) {
            float amount = (float)(n.player == p ? n.t_lose : n.t_win);
            fold_cfv(sp.hands[p], sp.hands[1 - p], reach_o, sp.same_combo[p], amount, out, sums);
        } else if (n.kind == K_SHOWDOWN) {
            showdown_cfv(sp.river_get(dealt), p, sp.hands[p], sp.hands[1 - p], reach_o, sp.same_combo[p],
                         (float)n.t_win, (float)n.t_lose, (float)n.t_tie, out, sums);
        } else if (n.kind == K_CHANCE) {
            std::vector<float> dummy(h, 1.0f);
            chance_node(n, p, dummy.data(), reach_o, dealt, out,
                        [&](uint32_t c, const float*, const float* ro, const Dealt& dd, float* o) {
                            br_into(c, p, ro, dd, o, avg_mode);
                        });
        } else {
            int na = n.num_children;
            if (n.player == p) {
                std::vector<float> vals(h);
                auto it = locks.find(idx);
                if (avg_mode || it != locks.end()) {
                    std::vector<float> sig(na * h);
                    average_strategy_into(idx, n, sig.data());
                    for (int a = 0; a < na; a++) {
                        std::fill(vals.begin(), vals.end(), 0.0f);
                        br_into(child(n, a), p, reach_o, dealt, vals.data(), avg_mode);
                        for (int i = 0; i < h; i++) out[i] += sig[a * h + i] * vals[i];
                    }
                } else {
                    for (int a = 0; a < na; a++) {
                        std::fill(vals.begin(), vals.end(), 0.0f);
                        br_into(child(n, a), p, reach_o, dealt, vals.data(), avg_mode);
                        if (a == 0) std::memcpy(out, vals.data(), sizeof(float) * h);
                        else for (int i = 0; i < h; i++) if (vals[i] > out[i]) out[i] = vals[i];
                    }
                }
            } else {
                std::vector<float> sig(na * ho), rb(ho), vals(h);
                average_strategy_into(idx, n, sig.data());
                for (int a = 0; a < na; a++) {
                    for (int j = 0; j < ho; j++) rb[j] = reach_o[j] * sig[a * ho + j];
                    std::fill(vals.begin(), vals.end(), 0.0f);
                    br_into(child(n, a), p, rb.data(), dealt, vals.data(), avg_mode);
                    for (int i = 0; i < h; i++) out[i] += vals[i];
                }
            }
        }
    }
    double pair_weight_sum() const {  // best_response.rs:227-251
        const auto& h0 = spot->hands[0];
        const auto& h1 = spot->hands[1];
        double t = 0, s[52] = {0};
        for (auto& h : h1) { double r = h.weight; t += r; s[h.c1] += r; s[h.c2] += r; }
        double total = 0;
        for (size_t i = 0; i < h0.size(); i++) {
            uint32_t same = spot->same_combo[0][i];
            double same_r = same != SENTINEL ? (double)h1[same].weight : 0.0;
            double valid = t - s[h0[i].c1] - s[h0[i].c2] + same_r;
            total += (double)h0[i].weight * valid;
        }
        return total;
    }
    double exploitability() {  // best_response.rs:255-287
        double denom = pair_weight_sum();
        if (denom <= 0.0) return NAN;
        double br[2];
        for (int p = 0; p < 2; p++) {
            std::vector<float> cfv(nh(p), 0.0f);
            br_into(0, p, spot->weights[1 - p].data(), Dealt(), cfv.data(), false);
            double acc = 0;
            for (int i = 0; i < nh(p); i++) acc += (double)spot->weights[p][i] * (double)cfv[i];
            br[p] = acc / denom;
        }
        if (spot->cfg.rake_pct > 0.0) {
            double v[2];
            for (int p = 0; p < 2; p++) {
                std::vector<float> cfv(nh(p), 0.0f);
                br_into(0, p, spot->weights[1 - p].data(), Dealt(), cfv.data(), true);
                double acc = 0;
                for (int i = 0; i < nh(p); i++) acc += (double)spot->weights[p][i] * (double)cfv[i];
                v[p] = acc / denom;
            }
            return ((br[0] - v[0]) + (br[1] - v[1])) / 2.0;
        }
        return (br[0] + br[1]) / 2.0;
    }

    // FP64 best-response oracle: the same traversal with every vector, strategy
    // and terminal sum in double (strategies normalised from the decoded arena).
    void avg_sigma64(uint32_t idx, const Node& n, double* sig) const {
        int p = n.player, h = nh(p), na = n.num_children;
        auto it = locks.find(idx);
        if (it != locks.end()) { for (int k = 0; k < na * h; k++) sig[k] = it->second[k]; return; }
        std::vector<float> s(na * h);
        strat[p].read_f32(idx, n.data_offset, na * h, s.data());
        for (int i = 0; i < h; i++) {
            double sum = 0;
            for (int a = 0; a < na; a++) sum += std::max<double>(s[a * h + i], 0.0);
            for (int a = 0; a < na; a++) sig[a * h + i] = sum > 1e-300 ? std::max<double>(s[a * h + i], 0.0) / sum : 1.0 / na;
        }
    }
    void br64(uint32_t idx, int p, const double* reach_o, const Dealt& dealt, double* out, bool avg_mode) {
        int ho = nh(1 - p), h = nh(p);
        bool any = false;
        for (int j = 0; j < ho; j++) any |= reach_o[j] > 0.0;
        if (!any) return;
        const Node& n = node(idx);
        const Spot& sp = *spot;
        if (n.kind == K_FOLD) {
            fold_cfv64(sp.hands[p], sp.hands[1 - p], reach_o, sp.same_combo[p], n.player == p ? n.t_lose : n.t_win, out);
        } else if (n.kind == K_SHOWDOWN) {
            showdown_cfv64(sp.river_get(dealt), p, sp.hands[p], sp.hands[1 - p], reach_o, sp.same_combo[p], n.t_win,
                           n.t_lose, n.t_tie, out);
        } else if (n.kind == K_CHANCE) {
            std::vector<Card> cards;
            for (int c = 0; c < 52; c++)
                if (sp.tree.children[n.children_start + c] != SENTINEL && !dealt.contains((Card)c)) cards.push_back((Card)c);
            std::vector<std::vector<double>> res(cards.size());
            auto run = [&](size_t k) {
                Card c = cards[k];
                uint64_t cm = cmask(c);
                std::vector<double> ro(ho);
                for (int j = 0; j < ho; j++) ro[j] = (sp.hands[1 - p][j].mask & cm) ? 0.0 : reach_o[j];
                res[k].assign(h, 0.0);
                uint32_t ch = sp.tree.children[n.children_start + c];
                // non-representative branches are materialised by ensure_symmetric first
                br64(ch, p, ro.data(), dealt.push(c), res[k].data(), avg_mode);
            };
            bool parallel = !cards.empty() && node(sp.tree.children[n.children_start + cards[0]]).kind == K_ACTION;
#ifdef _OPENMP
            if (parallel && !omp_in_parallel() && omp_get_max_threads() > 1) {
#pragma omp parallel for schedule(dynamic, 1)
                for (long k = 0; k < (long)cards.size(); k++) run((size_t)k);
            } else
#endif
            {
                (void)parallel;
                for (size_t k = 0; k < cards.size(); k++) run(k);
            }
            for (size_t k = 0; k < cards.size(); k++) {
                uint64_t cm = cmask(cards[k]);
                for (int i = 0; i < h; i++) if (!(sp.hands[p][i].mask & cm)) out[i] += res[k][i];
            }
            double div = 46.0 - (double)n.street;
            for (int i = 0; i < h; i++) out[i] /= div;
        } else {
            int na = n.num_children;
            if (n.player == p) {
                std::vector<double> vals(h);
                bool locked = locks.count(idx) > 0;
                if (avg_mode || locked) {
                    std::vector<double> sig(na * h);
                    avg_sigma64(idx, n, sig.data());
                    for (int a = 0; a < na; a++) {
                        std::fill(vals.begin(), vals.end(), 0.0);
                        br64(child(n, a), p, reach_o, dealt, vals.data(), avg_mode);
                        for (int i = 0; i < h; i++) out[i] += sig[a * h + i] * vals[i];
                    }
                } else {
                    for (int a = 0; a < na; a++) {
                        std::fill(vals.begin(), vals.end(), 0.0);
                        br64(child(n, a), p, reach_o, dealt, vals.data(), avg_mode);
                        for (int i = 0; i < h; i++) out[i] = a == 0 ? vals[i] : std::max(out[i], vals[i]);
                    }
                }
            } else {
                std::vector<double> sig(na * ho), rb(ho), vals(h);
                avg_sigma64(idx, n, sig.data());
                for (int a = 0; a < na; a++) {
                    for (int j = 0; j < ho; j++) rb[j] = reach_o[j] * sig[a * ho + j];
                    std::fill(vals.begin(), vals.end(), 0.0);
                    br64(child(n, a), p, rb.data(), dealt, vals.data(), avg_mode);
                    for (int i = 0; i < h; i++) out[i] += vals[i];
                }
            }
        }
    }
    double exploitability_f64() {
        ensure_symmetric();
        double denom = pair_weight_sum();
        if (denom <= 0.0) return NAN;
        double br[2], v[2] = {0, 0};
        bool raked = spot->cfg.rake_pct > 0.0;
        for (int p = 0; p < 2; p++)
            for (int m = 0; m < (raked ? 2 : 1); m++) {
                std::vector<double> ro(spot->weights[1 - p].begin(), spot->weights[1 - p].end());
                std::vector<double> cfv(nh(p), 0.0);
                br64(0, p, ro.data(), Dealt(), cfv.data(), m == 1);
                double acc = 0;
                for (int i = 0; i < nh(p); i++) acc += (double)spot->weights[p][i] * cfv[i];
                (m == 0 ? br[p] : v[p]) = acc / denom;
            }
        if (raked) return ((br[0] - v[0]) + (br[1] - v[1])) / 2.0;
        return (br[0] + br[1]) / 2.0;
    }

    // ---------------------------------------- cfr.rs:749-871 (symmetrize)
    void ensure_symmetric() {
        if (!sym_dirty || !use_iso || spot->suit_perms.size() < 2) { sym_dirty = false; return; }
        symmetrize_node(0, Dealt());
        sym_dirty = false;
    }
    void symmetrize_node(uint32_t idx, const Dealt& dealt) {
        const Node& n = node(idx);
        const Spot& sp = *spot;
        if (n.kind == K_ACTION) {
            for (int a = 0; a < n.num_children; a++) symmetrize_node(child(n, a), dealt);
        } else if (n.kind == K_CHANCE) {
            std::vector<int> valid = sp.perms_fixing(dealt);
            struct O { Card c, rep; int k; };
            std::vector<O> orbit;
            for (int c = 0; c < 52; c++) {
                if (sp.tree.children[n.children_start + c] == SENTINEL || dealt.contains((Card)c)) continue;
                Card rep = (Card)c;
                int k_rep = 0;
                for (int k : valid) {
                    Card pc = permute_card((Card)c, sp.suit_perms[k]);
                    if (pc < rep) { rep = pc; k_rep = k; }
                }
                orbit.push_back({(Card)c, rep, k_rep});
            }
            for (auto& o : orbit)
                if (o.c == o.rep) symmetrize_node(sp.tree.children[n.children_start + o.c], dealt.push(o.c));
            for (auto& o : orbit)
                if (o.c != o.rep)
                    copy_branch(sp.tree.children[n.children_start + o.rep], sp.tree.children[n.children_start + o.c], o.k);
        }
    }
    void copy_branch(uint32_t si, uint32_t di, int k) {
        const Node& s = node(si);
        const Node& dn = node(di);
        const Spot& sp = *spot;
        if (s.kind == K_ACTION) {
            int p = s.player, h = nh(p), na = s.num_children, cnt = na * h;
            const auto& tbl = sp.hand_perm[p][k];
            auto it = locks.find(si);
            std::vector<float> sr(cnt), ss(cnt), dr(cnt), ds(cnt);
            regrets[p].read_f32(si, s.data_offset, cnt, sr.data());
            strat[p].read_f32(si, s.data_offset, cnt, ss.data());
            for (int a = 0; a < na; a++)
                for (int i = 0; i < h; i++) {
                    int j = tbl[i];
                    dr[a * h + i] = sr[a * h + j];
                    ds[a * h + i] = it != locks.end() ? it->second[a * h + j] : ss[a * h + j];
                }
            regrets[p].write_f32(di, dn.data_offset, cnt, dr.data());
            strat[p].write_f32(di, dn.data_offset, cnt, ds.data());
            for (int a = 0; a < na; a++) copy_branch(child(s, a), child(dn, a), k);
        } else if (s.kind == K_CHANCE) {
            for (int x = 0; x < 52; x++) {
                uint32_t dc = sp.tree.children[dn.children_start + x];
                if (dc == SENTINEL) continue;
                Card sx = permute_card((Card)x, sp.suit_perms[k]);
                copy_branch(sp.tree.children[s.children_start + sx], dc, k);
            }
        }
    }
};

// --------------------------------------------------- query.rs lock creation
static bool normalize_freqs(const float* f, int n, int na, std::vector<float>& out) {  // query.rs:40-61
    if (n != na) { g_err = "expected action frequencies count mismatch"; return false; }
    for (int i = 0; i < n; i++) if (f[i] < 0.0f || !std::isfinite(f[i])) { g_err = "frequencies must be finite and >= 0"; return false; }
    double sum = 0;
    for (int i = 0; i < n; i++) sum += (double)f[i];
    if (!std::isfinite(sum) || sum > 1e9) { g_err = "frequencies sum is not a frequency vector"; return false; }
    if (sum <= 1e-9) { g_err = "at least one frequency must be positive"; return false; }
    out.resize(n);
    for (int i = 0; i < n; i++) out[i] = (float)((double)f[i] / sum);
    return true;
}
static void rake_to_target(float* sigma, int na, int nh, const float* reach, const float* target) {  // query.rs:68-156
    std::vector<double> m(na, 0.0);
    for (int a = 0; a < na; a++) if (target[a] > 1e-9f) m[a] = 1.0;
    for (int i = 0; i < nh; i++) {
        double mass = 0;
        for (int a = 0; a < na; a++) if (target[a] > 1e-9f) mass += (double)sigma[a * nh + i];
        if (mass <= 1e-12) for (int a = 0; a < na; a++) sigma[a * nh + i] = target[a];
    }
    for (int iter = 0; iter < 400; iter++) {
        std::vector<double> agg(na, 0.0);
        double total = 0;
        for (int i = 0; i < nh; i++) {
            double w = reach[i];
            if (w <= 0.0) continue;
            double denom = 0;
            for (int a = 0; a < na; a++) denom += m[a] * (double)sigma[a * nh + i];
            if (denom <= 1e-12) continue;
            total += w;
            for (int a = 0; a < na; a++) agg[a] += w * m[a] * (double)sigma[a * nh + i] / denom;
        }
        if (total <= 1e-12) break;
        double max_err = 0;
        for (int a = 0; a < na; a++) {
            if (target[a] <= 1e-9f) continue;
            double f = agg[a] / total;
            max_err = std::max(max_err, std::fabs(f - (double)target[a]));
            if (f > 1e-9) m[a] *= (double)target[a] / f;
        }
        double msum = 0;
        for (double x : m) msum += x;
        if (msum > 1e-12) {
            double scale = (double)na / msum;
            for (int a = 0; a < na; a++) m[a] *= scale;
        }
        if (max_err < 1e-4) break;
    }
    for (int i = 0; i < nh; i++) {
        double s = 0;
        for (int a = 0; a < na; a++) {
            double v = m[a] * (double)sigma[a * nh + i];
            sigma[a * nh + i] = (float)v;
            s += v;
        }
        if (s > 1e-12) {
            for (int a = 0; a < na; a++) sigma[a * nh + i] = (float)((double)sigma[a * nh + i] / s);
        } else {
            for (int a = 0; a < na; a++) sigma[a * nh + i] = target[a];
        }
    }
}

}  // namespace orc

// ------------------------------------------------------------------- C API
using namespace orc;
struct orc_spot { Spot* s; };
struct orc_solver { Solver* v; };

static TreeConfig to_cfg(const orc_config* c) {
    TreeConfig t;
    t.starting_pot = c->starting_pot;
    t.effective_stack = c->effective_stack;
    t.rake_pct = c->rake_pct;
    t.rake_cap = c->rake_cap;
    t.allin_threshold = c->allin_threshold;
    t.add_allin = c->add_allin != 0;
    t.max_raises = c->max_raises;
    for (int p = 0; p < 2; p++)
        for (int s = 0; s < 3; s++) {
            Sizing& z = p == 0 ? t.oop[s] : t.ip[s];
            std::vector<Size>* lists[3] = {&z.bet, &z.raise, &z.donk};
            for (int l = 0; l < 3; l++)
                for (int k = 0; k < c->n[p][s][l]; k++)
                    lists[l]->push_back({c->sizes[p][s][l][k].kind, c->sizes[p][s][l][k].value});
        }
    return t;
}

#define GUARD_BEGIN try {
#define GUARD_END(ret) } catch (const Err& e) { g_err = e.msg; return ret; } catch (const std::exception& e) { g_err = e.what(); return ret; }

extern "C" {
const char* orc_last_error(void) { return g_err.c_str(); }
void orc_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}
int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
uint32_t orc_evaluate7(const uint8_t* c) { return evaluate7(c); }
void orc_ref_eval7(const uint8_t* c, uint32_t* cat, uint8_t* ranks, int* nranks) {
    RefVal v = ref_eval7(c);
    *cat = v.cat;
    *nranks = (int)v.r.size();
    for (size_t i = 0; i < v.r.size(); i++) ranks[i] = v.r[i];
}
int orc_straight_top(uint16_t m) { return straight_top(m); }
int orc_combo_index(int a, int b) { return combo_index((Card)a, (Card)b); }
void orc_combo_from_index(int idx, int* hi, int* lo) {
    Card h, l;
    combo_from_index(idx, &h, &l);
    *hi = h;
    *lo = l;
}
int orc_parse_range(const char* s, float* w) {
    GUARD_BEGIN
    auto v = parse_range(s);
    std::memcpy(w, v.data(), sizeof(float) * 1326);
    return 0;
    GUARD_END(-1)
}
int orc_parse_cards(const char* s, uint8_t* out, int cap) {
    GUARD_BEGIN
    auto v = parse_cards(s);
    for (size_t i = 0; i < v.size() && (int)i < cap; i++) out[i] = v[i];
    return (int)v.size();
    GUARD_END(-1)
}
static int flops_out(const std::vector<std::pair<std::string, uint32_t>>& v, char* b, uint32_t* w, int cap) {
    for (size_t i = 0; i < v.size() && (int)i < cap; i++) {
        std::memcpy(b + 6 * i, v[i].first.data(), 6);
        w[i] = v[i].second;
    }
    return (int)v.size();
}
int orc_canonical_flops(char* b, uint32_t* w, int cap) { return flops_out(canonical_flops(), b, w, cap); }
int orc_canonical_flops_subset(int n, char* b, uint32_t* w, int cap) {
    return flops_out(canonical_flops_subset((size_t)n), b, w, cap);
}
float orc_encode_i16(const float* s, int n, int16_t* d) { return encode_i16(s, n, d); }
float orc_encode_u16(const float* s, int n, uint16_t* d) { return encode_u16(s, n, d); }
void orc_decode_i16(const int16_t* q, int n, float sc, float* o) { decode_i16(q, n, sc, o); }
void orc_decode_u16(const uint16_t* q, int n, float sc, float* o) { decode_u16(q, n, sc, o); }

orc_spot* orc_spot_new(const orc_config* cfg, int lenient, uint64_t max_nodes) {
    GUARD_BEGIN
    Spot* s = new_spot(to_cfg(cfg), cfg->board, cfg->range_oop, cfg->range_ip, max_nodes, lenient != 0);
    return new orc_spot{s};
    GUARD_END(nullptr)
}
void orc_spot_free(orc_spot* s) {
    if (s) { delete s->s; delete s; }
}
int64_t orc_spot_num_nodes(const orc_spot* s) { return (int64_t)s->s->tree.nodes.size(); }
int64_t orc_spot_num_children(const orc_spot* s) { return (int64_t)s->s->tree.children.size(); }
int64_t orc_spot_num_actions(const orc_spot* s) { return (int64_t)s->s->tree.actions.size(); }
int orc_spot_num_hands(const orc_spot* s, int p) { return (int)s->s->hands[p].size(); }
uint64_t orc_spot_data_size(const orc_spot* s, int p) { return s->s->tree.data_size[p]; }
int orc_spot_num_perms(const orc_spot* s) { return (int)s->s->suit_perms.size(); }
void orc_spot_nodes(const orc_spot* s, uint8_t* kind, uint8_t* player, uint8_t* street, uint8_t* nchild,
                    uint32_t* cs, uint32_t* as, uint64_t* doff, double* p0, double* p1, double* tw, double* tl,
                    double* tt) {
    const auto& nodes = s->s->tree.nodes;
    for (size_t i = 0; i < nodes.size(); i++) {
        const Node& n = nodes[i];
        if (kind) kind[i] = n.kind;
        if (player) player[i] = n.player;
        if (street) street[i] = n.street;
        if (nchild) nchild[i] = n.num_children;
        if (cs) cs[i] = n.children_start;
        if (as) as[i] = n.actions_start;
        if (doff) doff[i] = n.data_offset;
        if (p0) p0[i] = n.put[0];
        if (p1) p1[i] = n.put[1];
        if (tw) tw[i] = n.t_win;
        if (tl) tl[i] = n.t_lose;
        if (tt) tt[i] = n.t_tie;
    }
}
void orc_spot_children(const orc_spot* s, uint32_t* out) {
    std::memcpy(out, s->s->tree.children.data(), sizeof(uint32_t) * s->s->tree.children.size());
}
void orc_spot_actions(const orc_spot* s, int* kind, double* amount) {
    const auto& a = s->s->tree.actions;
    for (size_t i = 0; i < a.size(); i++) { kind[i] = a[i].kind; amount[i] = a[i].amount; }
}
void orc_spot_hands(const orc_spot* s, int p, uint8_t* c1, uint8_t* c2, float* w) {
    const auto& h = s->s->hands[p];
    for (size_t i = 0; i < h.size(); i++) { c1[i] = h[i].c1; c2[i] = h[i].c2; w[i] = h[i].weight; }
}
void orc_spot_same_combo(const orc_spot* s, int p, uint32_t* out) {
    std::memcpy(out, s->s->same_combo[p].data(), sizeof(uint32_t) * s->s->same_combo[p].size());
}
void orc_spot_perms(const orc_spot* s, uint8_t* perms4, uint16_t* hp0, uint16_t* hp1) {
    const Spot& sp = *s->s;
    for (size_t k = 0; k < sp.suit_perms.size(); k++) {
        for (int j = 0; j < 4; j++) perms4[4 * k + j] = sp.suit_perms[k][j];
        if (hp0) std::memcpy(hp0 + k * sp.hands[0].size(), sp.hand_perm[0][k].data(), 2 * sp.hands[0].size());
        if (hp1) std::memcpy(hp1 + k * sp.hands[1].size(), sp.hand_perm[1][k].data(), 2 * sp.hands[1].size());
    }
}
int orc_spot_river(const orc_spot* s, int p, const uint8_t* dealt, int nd, uint32_t* str, uint16_t* idx) {
    GUARD_BEGIN
    Dealt d;
    for (int i = 0; i < nd; i++) d = d.push(dealt[i]);
    const RiverEval& e = s->s->river_get(d);
    for (size_t k = 0; k < e.sorted[p].size(); k++) { str[k] = e.sorted[p][k].first; idx[k] = e.sorted[p][k].second; }
    return (int)e.sorted[p].size();
    GUARD_END(-1)
}
double orc_spot_pair_weight_sum(const orc_spot* s) {
    Solver tmp(s->s, false, DCFR, false, false);
    return tmp.pair_weight_sum();
}
void orc_fold_cfv(const orc_spot* s, int p, const float* ro, float amount, int exact, float* out) {
    fold_cfv(s->s->hands[p], s->s->hands[1 - p], ro, s->s->same_combo[p], amount, out, exact);
}
void orc_showdown_cfv(const orc_spot* s, int p, const uint8_t* dealt, int nd, const float* ro, float win, float lose,
                      float tie, int exact, float* out) {
    Dealt d;
    for (int i = 0; i < nd; i++) d = d.push(dealt[i]);
    showdown_cfv(s->s->river_get(d), p, s->s->hands[p], s->s->hands[1 - p], ro, s->s->same_combo[p], win, lose, tie, out,
                 exact);
}
void orc_fp8_encode(const float* x, int n, uint8_t* out) {
    for (int i = 0; i < n; i++) out[i] = f32_to_e4m3(x[i]);
}
void orc_fp8_decode(const uint8_t* q, int n, float* out) {
    for (int i = 0; i < n; i++) out[i] = e4m3_to_f32(q[i]);
}
orc_solver* orc_solver_new(orc_spot* s, int compressed, int algo, int use_iso, int prune) {
    return new orc_solver{new Solver(s->s, compressed, algo, use_iso != 0, prune != 0)};
}
void orc_solver_set_sums(orc_solver* v, int exact) { v->v->sums = exact ? 1 : 0; }
void orc_solver_set_rounding(orc_solver* v, int stochastic) { v->v->sr = stochastic ? 1 : 0; }
void orc_solver_free(orc_solver* v) {
    if (v) { delete v->v; delete v; }
}
void orc_solver_iterate(orc_solver* v, int n) {
    for (int i = 0; i < n; i++) v->v->iterate();
}
uint32_t orc_solver_iteration(const orc_solver* v) { return v->v->iteration; }
void orc_solver_set_iteration(orc_solver* v, uint32_t it) { v->v->iteration = it; }
double orc_solver_exploitability(orc_solver* v) { return v->v->exploitability(); }
double orc_solver_exploitability_f64(orc_solver* v) { return v->v->exploitability_f64(); }
static Store* pick(Solver* s, int which, int p) {
    if (which == 0) return &s->regrets[p];
    if (which == 1) return &s->strat[p];
    if (!s->have_preds) s->ensure_preds();
    return &s->preds[p];
}
int orc_solver_get_arena(const orc_solver* vc, int which, int p, float* out) {
    Solver* s = vc->v;
    Store* st = pick(s, which, p);
    int h = s->nh(p);
    std::memset(out, 0, sizeof(float) * s->spot->tree.data_size[p]);
    const auto& nodes = s->spot->tree.nodes;
    for (size_t i = 0; i < nodes.size(); i++)
        if (nodes[i].kind == K_ACTION && nodes[i].player == p)
            st->read_f32((uint32_t)i, nodes[i].data_offset, nodes[i].num_children * h, out + nodes[i].data_offset);
    return 0;
}
int orc_solver_set_arena(orc_solver* vc, int which, int p, const float* in) {
    Solver* s = vc->v;
    Store* st = pick(s, which, p);
    int h = s->nh(p);
    const auto& nodes = s->spot->tree.nodes;
    for (size_t i = 0; i < nodes.size(); i++)
        if (nodes[i].kind == K_ACTION && nodes[i].player == p)
            st->write_f32((uint32_t)i, nodes[i].data_offset, nodes[i].num_children * h, in + nodes[i].data_offset);
    return 0;
}
int orc_solver_set_lock(orc_solver* v, uint32_t node, const float* sigma, int n) {
    v->v->locks[node] = std::vector<float>(sigma, sigma + n);
    v->v->sym_dirty = true;
    return 0;
}
void orc_solver_clear_locks(orc_solver* v) { v->v->locks.clear(); }
int orc_solver_avg_strategy(const orc_solver* v, uint32_t node, float* out) {
    v->v->average_strategy_into(node, v->v->node(node), out);
    return 0;
}
int orc_solver_solved_strategy(const orc_solver* v, uint32_t node, float* out) {
    v->v->solved_strategy_into(v->v->node(node), out);
    return 0;
}
void orc_solver_ensure_symmetric(orc_solver* v) { v->v->ensure_symmetric(); }
void orc_solver_root_br_cfv(orc_solver* v, int p, float* out) {
    std::fill(out, out + v->v->nh(p), 0.0f);
    v->v->br_into(0, p, v->v->spot->weights[1 - p].data(), Dealt(), out, false);
}
void orc_solver_discounts(int algo, uint32_t t, float* pos, float* neg, float* strat) {
    Disc d = discounts(algo, t);
    *pos = d.pos;
    *neg = d.neg;
    *strat = d.strat;
}
int orc_solver_walk_path(orc_solver* vc, const int* steps, int ns, uint32_t* node_out, float* r0, float* r1) {
    // query.rs:304-340 (walk_path), on an already-canonical path
    GUARD_BEGIN
    Solver* s = vc->v;
    const Spot& sp = *s->spot;
    uint32_t ni = 0;
    std::vector<float> reach[2] = {sp.weights[0], sp.weights[1]};
    Dealt dealt;
    for (int k = 0; k < ns; k++) {
        const Node& n = s->node(ni);
        if (n.kind == K_ACTION && steps[k] >= 0) {
            int idx = steps[k], na = n.num_children;
            if (idx >= na) fail("action index out of range");
            int p = n.player, h = s->nh(p);
            std::vector<float> sig(na * h);
            s->average_strategy_into(ni, n, sig.data());
            for (int i = 0; i < h; i++) reach[p][i] *= sig[idx * h + i];
            ni = sp.tree.children[n.children_start + idx];
        } else if (n.kind == K_CHANCE && steps[k] < 0) {
            Card c = (Card)(-1 - steps[k]);
            uint32_t ch = sp.tree.children[n.children_start + c];
            if (ch == SENTINEL || dealt.contains(c)) fail("card not available here");
            for (int p = 0; p < 2; p++)
                for (size_t i = 0; i < sp.hands[p].size(); i++)
                    if (sp.hands[p][i].mask & cmask(c)) reach[p][i] = 0.0f;
            dealt = dealt.push(c);
            ni = ch;
        } else {
            fail("path step does not match node kind");
        }
    }
    *node_out = ni;
    if (r0) std::memcpy(r0, reach[0].data(), sizeof(float) * reach[0].size());
    if (r1) std::memcpy(r1, reach[1].data(), sizeof(float) * reach[1].size());
    return 0;
    GUARD_END(-1)
}
int orc_solver_node_values(orc_solver* vc, const int* steps, int ns, int p, int avg, float* cfv, float* child_cfv,
                           float* r0, float* r1) {
    // query.rs:490-600 (node_view's traversals): walk_path (query.rs:304-340),
    // then traverse_avg (avg = 1, best_response.rs:128-223) or traverse_br
    // (avg = 0, best_response.rs:19-124) of the node for player p with the
    // opponent's walk reach, and of each child when p acts there
    GUARD_BEGIN
    Solver* s = vc->v;
    const Spot& sp = *s->spot;
    uint32_t ni = 0;
    std::vector<float> reach[2] = {sp.weights[0], sp.weights[1]};
    Dealt dealt;
    for (int k = 0; k < ns; k++) {
        const Node& n = s->node(ni);
        if (n.kind == K_ACTION && steps[k] >= 0) {
            int idx = steps[k], na = n.num_children;
            if (idx >= na) fail("action index out of range");
            int q = n.player, h = s->nh(q);
            std::vector<float> sig(na * h);
            s->average_strategy_into(ni, n, sig.data());
            for (int i = 0; i < h; i++) reach[q][i] *= sig[idx * h + i];
            ni = sp.tree.children[n.children_start + idx];
        } else if (n.kind == K_CHANCE && steps[k] < 0) {
            Card c = (Card)(-1 - steps[k]);
            uint32_t ch = sp.tree.children[n.children_start + c];
            if (ch == SENTINEL || dealt.contains(c)) fail("card not available here");
            for (int q = 0; q < 2; q++)
                for (size_t i = 0; i < sp.hands[q].size(); i++)
                    if (sp.hands[q][i].mask & cmask(c)) reach[q][i] = 0.0f;
            dealt = dealt.push(c);
            ni = ch;
        } else {
            fail("path step does not match node kind");
        }
    }
    const int h = s->nh(p);
    const float* ro = reach[1 - p].data();
    std::fill(cfv, cfv + h, 0.0f);
    s->br_into(ni, p, ro, dealt, cfv, avg != 0);
    const Node& n = s->node(ni);
    if (child_cfv && n.kind == K_ACTION && n.player == p)
        for (int a = 0; a < n.num_children; a++) {
            std::fill(child_cfv + (size_t)a * h, child_cfv + (size_t)(a + 1) * h, 0.0f);
            s->br_into(sp.tree.children[n.children_start + a], p, ro, dealt, child_cfv + (size_t)a * h, avg != 0);
        }
    if (r0) std::memcpy(r0, reach[0].data(), sizeof(float) * reach[0].size());
    if (r1) std::memcpy(r1, reach[1].data(), sizeof(float) * reach[1].size());
    return (int)ni;
    GUARD_END(-1)
}
void orc_rake_to_target(float* sigma, int na, int nh, const float* reach, const float* target) {
    rake_to_target(sigma, na, nh, reach, target);
}
int orc_normalize_freqs(const float* f, int n, float* out) {
    std::vector<float> v;
    if (!normalize_freqs(f, n, n, v)) return -1;
    std::memcpy(out, v.data(), sizeof(float) * n);
    return 0;
}
int orc_solver_lock_node(orc_solver* vc, const int* steps, int ns, int mode, const float* freqs, int nf,
                         const char* combo) {
    // query.rs:700-773 on a canonical path (mode 0 freeze, 1 range, 2 one hand edit)
    GUARD_BEGIN
    Solver* s = vc->v;
    const Spot& sp = *s->spot;
    uint32_t ni;
    std::vector<float> r0(sp.hands[0].size()), r1(sp.hands[1].size());
    if (orc_solver_walk_path(vc, steps, ns, &ni, r0.data(), r1.data()) != 0) return -1;
    const Node& n = s->node(ni);
    if (n.kind != K_ACTION) fail("only action nodes can be locked");
    int na = n.num_children, p = n.player, h = s->nh(p);
    std::vector<float> sig(na * h);
    if (mode == 0) {
        s->solved_strategy_into(n, sig.data());
    } else if (mode == 1) {
        std::vector<float> tgt;
        if (!normalize_freqs(freqs, nf, na, tgt)) return -1;
        s->solved_strategy_into(n, sig.data());
        rake_to_target(sig.data(), na, h, p == 0 ? r0.data() : r1.data(), tgt.data());
    } else {
        std::vector<float> tgt;
        if (!normalize_freqs(freqs, nf, na, tgt)) return -1;
        s->average_strategy_into(ni, n, sig.data());
        auto cards = parse_cards(combo);
        if (cards.size() != 2) fail("expected a 2-card combo");
        int idx = -1;
        for (int i = 0; i < h; i++) {
            const Hand& hd = sp.hands[p][i];
            if ((hd.c1 == cards[0] && hd.c2 == cards[1]) || (hd.c1 == cards[1] && hd.c2 == cards[0])) { idx = i; break; }
        }
        if (idx < 0) fail("combo is not in range here");
        for (int a = 0; a < na; a++) sig[a * h + idx] = tgt[a];
    }
    s->locks[ni] = sig;
    s->sym_dirty = true;
    return (int)ni;
    GUARD_END(-1)
}
}  // extern "C"
