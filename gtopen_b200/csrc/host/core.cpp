// Host model of a spot: see core.hpp.  Citations are to the reference solver
// crate (crates/solver/src/...).
#include "core.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <unordered_map>

namespace gtob {

static const char kRankCh[] = "23456789TJQKA";
static const char kSuitCh[] = "cdhs";

static std::string strip(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\n\r\f\v");
    if (a == std::string::npos) return std::string();
    size_t b = s.find_last_not_of(" \t\n\r\f\v");
    return s.substr(a, b - a + 1);
}
static int rank_index(char c) {
    const char* p = strchr(kRankCh, toupper((unsigned char)c));
    return (p && c) ? (int)(p - kRankCh) : -1;
}
static int suit_index(char c) {
    const char* p = strchr(kSuitCh, tolower((unsigned char)c));
    return (p && c) ? (int)(p - kSuitCh) : -1;
}

// cards.rs:106-114
void combo_cards(int id, uint8_t* hi, uint8_t* lo) {
    int h = 1;
    while ((h + 1) * h / 2 <= id) ++h;
    *hi = (uint8_t)h;
    *lo = (uint8_t)(id - h * (h - 1) / 2);
}
// cards.rs:47-55
uint8_t parse_card(const std::string& s0) {
    std::string s = strip(s0);
    if (s.size() != 2) throw Error("invalid card: \"" + s0 + "\"");
    int r = rank_index(s[0]), su = suit_index(s[1]);
    if (r < 0) throw Error("invalid rank in card: \"" + s0 + "\"");
    if (su < 0) throw Error("invalid suit in card: \"" + s0 + "\"");
    return card_make(r, su);
}
// cards.rs:66-86
std::vector<uint8_t> parse_board(const std::string& s) {
    std::string cl;
    for (char c : s)
        if (!isspace((unsigned char)c) && c != ',') cl += c;
    if (cl.size() & 1) throw Error("invalid card list: \"" + s + "\"");
    std::vector<uint8_t> out;
    uint64_t seen = 0;
    for (size_t i = 0; i + 1 < cl.size(); i += 2) {
        uint8_t c = parse_card(cl.substr(i, 2));
        if ((seen >> c) & 1) throw Error("duplicate card in list: \"" + s + "\"");
        seen |= 1ull << c;
        out.push_back(c);
    }
    return out;
}
std::string card_name(uint8_t c) { return std::string{kRankCh[card_rank(c)], kSuitCh[card_suit(c)]}; }

// ---------------------------------------------------------------- evaluator
// evaluator.rs:68-175.  Value = category << 20 | five 4-bit tiebreak ranks.
static inline uint32_t pack(uint32_t cat, int r0 = 0, int r1 = 0, int r2 = 0, int r3 = 0, int r4 = 0) {
    return (cat << 20) | ((uint32_t)r0 << 16) | ((uint32_t)r1 << 12) | ((uint32_t)r2 << 8) | ((uint32_t)r3 << 4) |
           (uint32_t)r4;
}
// Highest straight top in a 13-bit rank mask (wheel = 3), or -1
// (evaluator.rs:33-49): a run of five set bits in the mask with the ace
// copied below the deuce.
static inline int best_straight(uint32_t rm) {
    uint32_t m = (rm << 1) | ((rm >> 12) & 1u);
    uint32_t run = m & (m >> 1) & (m >> 2) & (m >> 3) & (m >> 4);
    if (!run) return -1;
    return 31 - __builtin_clz(run) + 3;
}
// Highest n set ranks of a mask, most significant first (evaluator.rs:53-65).
static inline void highest(uint32_t rm, int n, int* out) {
    for (int k = 0; k < n; k++) out[k] = 0;
    for (int k = 0; k < n && rm; k++) {
        int r = 31 - __builtin_clz(rm);
        out[k] = r;
        rm &= ~(1u << r);
    }
}
uint32_t eval7(const uint8_t* cards) {
    uint32_t by_suit[4] = {0, 0, 0, 0};
    int cnt[13] = {0};
    for (int k = 0; k < 7; k++) {
        by_suit[cards[k] & 3] |= 1u << (cards[k] >> 2);
        cnt[cards[k] >> 2]++;
    }
    uint32_t ranks = by_suit[0] | by_suit[1] | by_suit[2] | by_suit[3];
    int fs = -1;
    for (int s = 0; s < 4 && fs < 0; s++)
        if (__builtin_popcount(by_suit[s]) >= 5) fs = s;
    if (fs >= 0) {
        int t = best_straight(by_suit[fs]);
        if (t >= 0) return pack(8, t);
    }
    int quad = -1, trip[2] = {-1, -1}, pair[3] = {-1, -1, -1}, nt = 0, np = 0;
    for (int r = 12; r >= 0; r--) {
        if (cnt[r] == 4) quad = r;
        else if (cnt[r] == 3 && nt < 2) trip[nt++] = r;
        else if (cnt[r] == 2 && np < 3) pair[np++] = r;
    }
    int k[5];
    if (quad >= 0) {
        highest(ranks & ~(1u << quad), 1, k);
        return pack(7, quad, k[0]);
    }
    if (nt >= 1 && (nt >= 2 || np >= 1)) return pack(6, trip[0], nt >= 2 ? trip[1] : pair[0]);
    if (fs >= 0) {
        highest(by_suit[fs], 5, k);
        return pack(5, k[0], k[1], k[2], k[3], k[4]);
    }
    int st = best_straight(ranks);
    if (st >= 0) return pack(4, st);
    if (nt >= 1) {
        highest(ranks & ~(1u << trip[0]), 2, k);
        return pack(3, trip[0], k[0], k[1]);
    }
    if (np >= 2) {
        highest(ranks & ~(1u << pair[0]) & ~(1u << pair[1]), 1, k);
        return pack(2, pair[0], pair[1], k[0]);
    }
    if (np == 1) {
        highest(ranks & ~(1u << pair[0]), 3, k);
        return pack(1, pair[0], k[0], k[1], k[2]);
    }
    highest(ranks, 5, k);
    return pack(0, k[0], k[1], k[2], k[3], k[4]);
}

// -------------------------------------------------------------------- range
// range.rs: tokens separated by ',' or ' ' (after '\n' '\t' ';' -> ','),
// optional ':weight' (> 1 means percent), later tokens overwrite earlier.
namespace {
using ComboList = std::vector<std::pair<uint8_t, uint8_t>>;
void add_pair_class(int r, ComboList& out) {  // range.rs:144-152
    for (int s1 = 0; s1 < 4; s1++)
        for (int s2 = 0; s2 < s1; s2++) out.push_back({card_make(r, s1), card_make(r, s2)});
}
void add_suited(int hi, int lo, ComboList& out) {  // range.rs:154-161
    for (int s = 0; s < 4; s++) out.push_back({card_make(hi, s), card_make(lo, s)});
}
void add_offsuit(int hi, int lo, ComboList& out) {  // range.rs:162-173
    for (int s1 = 0; s1 < 4; s1++)
        for (int s2 = 0; s2 < 4; s2++)
            if (s1 != s2) out.push_back({card_make(hi, s1), card_make(lo, s2)});
}
void add_class(int hi, int lo, char marker, ComboList& out) {  // range.rs:178-200
    if (hi == lo) {
        if (marker) throw Error("pairs cannot have a suitedness marker");
        add_pair_class(hi, out);
        return;
    }
    if (marker == 's') add_suited(hi, lo, out);
    else if (marker == 'o') add_offsuit(hi, lo, out);
    else if (marker == 0) { add_suited(hi, lo, out); add_offsuit(hi, lo, out); }
    else throw Error("invalid suitedness marker");
}
struct Cls { int hi, lo; char m; };
bool read_class(const std::string& s, Cls* c) {  // range.rs:203-221
    if (s.size() != 2 && s.size() != 3) return false;
    int a = rank_index(s[0]), b = rank_index(s[1]);
    if (a < 0 || b < 0) return false;
    char m = 0;
    if (s.size() == 3) {
        m = (char)tolower((unsigned char)s[2]);
        if (m != 's' && m != 'o') return false;
    }
    *c = {std::max(a, b), std::min(a, b), m};
    return true;
}
ComboList expand(const std::string& raw) {  // range.rs:223-303
    std::string it = strip(raw);
    ComboList out;
    if (it.size() == 4 && rank_index(it[0]) >= 0 && suit_index(it[1]) >= 0 && rank_index(it[2]) >= 0 &&
        suit_index(it[3]) >= 0) {
        uint8_t a = parse_card(it.substr(0, 2)), b = parse_card(it.substr(2, 2));
        if (a == b) throw Error("combo with duplicate card: \"" + it + "\"");
        out.push_back({a, b});
        return out;
    }
    size_t dash = it.find('-');
    if (dash != std::string::npos) {
        Cls x, y;
        if (!read_class(strip(it.substr(0, dash)), &x)) throw Error("invalid range start: \"" + it + "\"");
        if (!read_class(strip(it.substr(dash + 1)), &y)) throw Error("invalid range end: \"" + it + "\"");
        if (x.m != y.m) throw Error("mismatched suitedness in range: \"" + it + "\"");
        if (x.hi == x.lo && y.hi == y.lo) {
            for (int r = std::min(x.hi, y.hi); r <= std::max(x.hi, y.hi); r++) add_class(r, r, x.m, out);
        } else if (x.hi == y.hi) {
            for (int r = std::min(x.lo, y.lo); r <= std::max(x.lo, y.lo); r++)
                if (r != x.hi) add_class(x.hi, r, x.m, out);
        } else if (x.hi - x.lo == y.hi - y.lo) {
            int gap = x.hi - x.lo;
            for (int h = std::min(x.hi, y.hi); h <= std::max(x.hi, y.hi); h++) add_class(h, h - gap, x.m, out);
        } else {
            throw Error("unsupported range shape: \"" + it + "\"");
        }
        return out;
    }
    if (!it.empty() && it.back() == '+') {
        Cls x;
        if (!read_class(strip(it.substr(0, it.size() - 1)), &x)) throw Error("invalid item: \"" + it + "\"");
        if (x.hi == x.lo)
            for (int r = x.hi; r < 13; r++) add_class(r, r, x.m, out);
        else
            for (int l = x.lo; l < x.hi; l++) add_class(x.hi, l, x.m, out);
        return out;
    }
    Cls x;
    if (!read_class(it, &x)) throw Error("invalid range token: \"" + it + "\"");
    add_class(x.hi, x.lo, x.m, out);
    return out;
}
}  // namespace

std::vector<float> parse_range_weights(const std::string& text) {  // range.rs:28-58
    std::vector<float> w(1326, 0.0f);
    std::string s = text;
    for (auto& c : s)
        if (c == '\n' || c == '\t' || c == ';') c = ',';
    size_t pos = 0;
    for (;;) {
        size_t end = s.find_first_of(", ", pos);
        std::string tok = strip(s.substr(pos, end == std::string::npos ? std::string::npos : end - pos));
        if (!tok.empty()) {
            float weight = 1.0f;
            std::string item = tok;
            size_t c = tok.rfind(':');
            if (c != std::string::npos) {
                item = strip(tok.substr(0, c));
                std::string ws = strip(tok.substr(c + 1));
                char* e = nullptr;
                weight = strtof(ws.c_str(), &e);
                if (ws.empty() || *e) throw Error("invalid weight in token \"" + tok + "\"");
                if (weight > 1.0f) weight /= 100.0f;
                if (!(weight >= 0.0f && weight <= 1.0f)) throw Error("weight out of range in token \"" + tok + "\"");
            }
            for (auto& pr : expand(item)) w[combo_id(pr.first, pr.second)] = weight;
        }
        if (end == std::string::npos) break;
        pos = end + 1;
    }
    return w;
}

// ------------------------------------------------------------------- config
static std::vector<BetSize> sizes_from(const json::Value* v) {
    std::vector<BetSize> out;
    if (!v || v->kind == json::Value::NUL) return out;
    if (v->kind != json::Value::ARR) throw Error("size list must be an array");
    for (auto& e : v->arr) {
        if (e.kind == json::Value::STR && e.str == "AllIn") { out.push_back({kAllIn, 0.0}); continue; }
        if (e.kind == json::Value::OBJ && e.obj.size() == 1 && e.obj[0].second.kind == json::Value::NUM) {
            if (e.obj[0].first == "PotPct") { out.push_back({kPotPct, e.obj[0].second.num}); continue; }
            if (e.obj[0].first == "PrevMult") { out.push_back({kPrevMult, e.obj[0].second.num}); continue; }
        }
        throw Error("unknown bet size entry");
    }
    return out;
}
static double num_or(const json::Value& o, const char* k, double dflt, bool required) {
    const json::Value* v = o.get(k);
    if (!v) {
        if (required) throw Error(std::string("missing field `") + k + "`");
        return dflt;
    }
    if (v->kind != json::Value::NUM) throw Error(std::string("field `") + k + "` must be a number");
    return v->num;
}
static std::string str_of(const json::Value& o, const char* k) {
    const json::Value* v = o.get(k);
    if (!v || v->kind != json::Value::STR) throw Error(std::string("missing string field `") + k + "`");
    return v->str;
}
SpotConfig config_from_json(const json::Value& v) {
    if (v.kind != json::Value::OBJ) throw Error("spot config must be a JSON object");
    SpotConfig c;
    c.board = str_of(v, "board");
    c.range_oop = str_of(v, "range_oop");
    c.range_ip = str_of(v, "range_ip");
    const json::Value* t = v.get("tree");
    if (!t || t->kind != json::Value::OBJ) throw Error("missing field `tree`");
    TreeConfig& tc = c.tree;
    tc.starting_pot = num_or(*t, "starting_pot", 0, true);
    tc.effective_stack = num_or(*t, "effective_stack", 0, true);
    tc.rake_pct = num_or(*t, "rake_pct", 0.0, false);
    tc.rake_cap = num_or(*t, "rake_cap", 0.0, false);
    tc.allin_threshold = num_or(*t, "allin_threshold", 0.85, false);
    tc.max_raises = (int)num_or(*t, "max_raises", 10, false);
    const json::Value* aa = t->get("add_allin");
    tc.add_allin = aa && aa->kind == json::Value::BOOL && aa->b;
    for (int p = 0; p < 2; p++) {
        const json::Value* arr = t->get(p == 0 ? "oop" : "ip");
        if (!arr || arr->kind != json::Value::ARR || arr->arr.size() != 3)
            throw Error(std::string("field `") + (p == 0 ? "oop" : "ip") + "` must hold 3 street sizings");
        for (int s = 0; s < 3; s++) {
            StreetSizing& z = p == 0 ? tc.oop[s] : tc.ip[s];
            const json::Value& o = arr->arr[s];
            z.bet = sizes_from(o.get("bet"));
            z.raise = sizes_from(o.get("raise"));
            z.donk = sizes_from(o.get("donk"));
        }
    }
    return c;
}
static json::Value sizes_to(const std::vector<BetSize>& l) {
    json::Value a = json::Value::array();
    for (auto& s : l) {
        if (s.kind == kAllIn) { a.arr.push_back(json::Value::string("AllIn")); continue; }
        json::Value o = json::Value::object();
        o.set(s.kind == kPotPct ? "PotPct" : "PrevMult", json::Value::number(s.v));
        a.arr.push_back(o);
    }
    return a;
}
json::Value config_to_json(const SpotConfig& c) {
    json::Value t = json::Value::object();
    const TreeConfig& tc = c.tree;
    t.set("starting_pot", json::Value::number(tc.starting_pot));
    t.set("effective_stack", json::Value::number(tc.effective_stack));
    t.set("rake_pct", json::Value::number(tc.rake_pct));
    t.set("rake_cap", json::Value::number(tc.rake_cap));
    for (int p = 0; p < 2; p++) {
        json::Value arr = json::Value::array();
        for (int s = 0; s < 3; s++) {
            const StreetSizing& z = p == 0 ? tc.oop[s] : tc.ip[s];
            json::Value o = json::Value::object();
            o.set("bet", sizes_to(z.bet)).set("raise", sizes_to(z.raise)).set("donk", sizes_to(z.donk));
            arr.arr.push_back(o);
        }
        t.set(p == 0 ? "oop" : "ip", arr);
    }
    t.set("allin_threshold", json::Value::number(tc.allin_threshold));
    t.set("add_allin", json::Value::boolean(tc.add_allin));
    json::Value mr = json::Value::integer(tc.max_raises);
    t.set("max_raises", mr);
    json::Value v = json::Value::object();
    v.set("board", json::Value::string(c.board));
    v.set("range_oop", json::Value::string(c.range_oop));
    v.set("range_ip", json::Value::string(c.range_ip));
    v.set("tree", t);
    return v;
}

// --------------------------------------------------------------------- tree
namespace {
struct St {  // betting state while building (tree.rs:213-224)
    int street, actor;
    double put[2], bet[2], last_inc;
    int raises, aggressor;  // aggressor -1 = none
    bool checked;
};
void sort_dedupe(std::vector<double>& v) {  // tree.rs:781-787
    std::stable_sort(v.begin(), v.end());
    size_t w = 0;
    for (size_t r = 0; r < v.size(); r++)
        if (w == 0 || !(std::fabs(v[r] - v[w - 1]) < 1e-6)) v[w++] = v[r];
    v.resize(w);
}
class Builder {
  public:
    Builder(const TreeConfig& c, int rs, uint64_t bm, uint64_t cap, uint64_t nh0, uint64_t nh1)
        : c_(c), rs_(rs), bm_(bm), cap_(cap) {
        nh_[0] = nh0;
        nh_[1] = nh1;
        t_.root_street = rs;
    }
    Tree take() { return std::move(t_); }
    uint32_t decision(const St& st) {  // tree.rs:535-574
        budget();
        std::vector<std::pair<uint8_t, double>> acts = legal(st);
        if (acts.empty() || acts.size() > 250) throw Error("invalid action count during tree build");
        uint32_t id = add(kAction, (uint8_t)st.actor, (uint8_t)st.street, st.put);
        t_.nchild[id] = (uint8_t)acts.size();
        t_.action_start[id] = (uint32_t)t_.act_kind.size();
        for (auto& a : acts) { t_.act_kind.push_back(a.first); t_.act_amount.push_back(a.second); }
        t_.data_off[id] = t_.data_size[st.actor];
        t_.data_size[st.actor] += acts.size() * nh_[st.actor];
        std::vector<uint32_t> kids;
        kids.reserve(acts.size());
        for (auto& a : acts) kids.push_back(follow(st, a.first, a.second));
        t_.child_start[id] = (uint32_t)t_.children.size();
        t_.children.insert(t_.children.end(), kids.begin(), kids.end());
        return id;
    }

  private:
    const TreeConfig& c_;
    int rs_;
    uint64_t bm_, cap_, nh_[2];
    Tree t_;

    void budget() {  // tree.rs:412-420
        if (cap_ && t_.size() >= cap_)
            throw Error("tree too large: over the max_nodes budget of " + std::to_string(cap_) +
                        "; reduce bet/raise sizes, max_raises, or effective stack");
    }
    double rake(double pot) const {  // tree.rs:526-533
        double r = c_.rake_pct * pot;
        return c_.rake_cap > 0.0 ? std::min(r, c_.rake_cap) : r;
    }
    uint32_t add(uint8_t kind, uint8_t player, uint8_t street, const double* put) {
        t_.kind.push_back(kind);
        t_.player.push_back(player);
        t_.street.push_back(street);
        t_.nchild.push_back(0);
        t_.child_start.push_back(0);
        t_.action_start.push_back(0);
        t_.data_off.push_back(0);
        t_.put0.push_back(put[0]);
        t_.put1.push_back(put[1]);
        t_.twin.push_back(0.0);
        t_.tlose.push_back(0.0);
        t_.ttie.push_back(0.0);
        return (uint32_t)(t_.size() - 1);
    }
    // tree.rs:432-524
    std::vector<std::pair<uint8_t, double>> legal(const St& st) const {
        const int me = st.actor, op = 1 - me;
        const double stack = c_.effective_stack - (st.put[me] - c_.starting_pot / 2.0);
        const double facing = st.bet[op] - st.bet[me];
        const StreetSizing& sz = c_.side(st.actor, st.street);
        std::vector<std::pair<uint8_t, double>> out;
        std::vector<double> to;
        if (facing > 1e-9) {
            out.push_back({kFoldA, 0.0});
            out.push_back({kCall, st.bet[op]});
            if (!(stack > facing + 1e-9 && st.raises < c_.max_raises)) return out;
            const double pot_call = st.put[0] + st.put[1] + facing;
            const double cap = st.bet[me] + stack;
            std::vector<double> cand;
            for (const BetSize& b : sz.raise)
                cand.push_back(b.kind == kPotPct ? st.bet[op] + b.v / 100.0 * pot_call
                               : b.kind == kPrevMult ? st.bet[op] * b.v : cap);
            if (c_.add_allin) cand.push_back(cap);
            const double floor = st.bet[op] + std::max(st.last_inc, 1e-9);
            for (double x : cand) {
                if (x < floor) x = floor;
                if (x >= cap - 1e-9 || x >= c_.allin_threshold * cap - 1e-9) x = cap;
                if (x > st.bet[op] + 1e-9) to.push_back(x);
            }
            sort_dedupe(to);
            for (double x : to) out.push_back({kRaise, x});
            return out;
        }
        out.push_back({kCheck, 0.0});
        if (!(stack > 1e-9)) return out;
        const bool donk = st.actor == 0 && st.street > rs_ && st.aggressor == 1;
        const std::vector<BetSize>& list = donk ? sz.donk : sz.bet;
        const double pot = st.put[0] + st.put[1];
        std::vector<double> cand;
        for (const BetSize& b : list) {
            if (b.kind == kPrevMult) continue;  // dropped (lenient rebuilds of old saves)
            cand.push_back(b.kind == kPotPct ? b.v / 100.0 * pot : stack);
        }
        if (c_.add_allin && (!list.empty() || !donk)) cand.push_back(stack);
        for (double x : cand) {
            if (x <= 1e-9) continue;
            if (x >= stack - 1e-9 || x >= c_.allin_threshold * stack - 1e-9) x = stack;
            to.push_back(x);
        }
        sort_dedupe(to);
        for (double x : to) out.push_back({kBet, x});
        return out;
    }
    // tree.rs:576-652
    uint32_t follow(const St& st, uint8_t kind, double amt) {
        const int me = st.actor, op = 1 - me;
        switch (kind) {
            case kFoldA: {
                double f = st.put[me];
                double rk = rake(2.0 * f);
                uint32_t id = add(kFold, (uint8_t)st.actor, (uint8_t)st.street, st.put);
                t_.twin[id] = f - rk;
                t_.tlose[id] = -f;
                return id;
            }
            case kCheck: {
                if (st.checked) return street_over(st.street, st.put, st.aggressor, false);
                St n = st;
                n.actor ^= 1;
                n.checked = true;
                return decision(n);
            }
            case kCall: {
                double put[2] = {st.put[0], st.put[1]};
                put[me] += amt - st.bet[me];
                double half = c_.starting_pot / 2.0;
                bool allin = c_.effective_stack - (put[me] - half) <= 1e-9 || c_.effective_stack - (put[op] - half) <= 1e-9;
                return street_over(st.street, put, st.actor ^ 1, allin);
            }
            default: {
                St n = st;
                n.put[me] += amt - st.bet[me];
                n.bet[me] = amt;
                n.actor ^= 1;
                n.last_inc = std::max(amt - std::max(st.bet[op], st.bet[me]), st.last_inc);
                n.raises = st.raises + (kind == kRaise ? 1 : 0);
                return decision(n);
            }
        }
    }
    // tree.rs:662-723
    uint32_t street_over(int street, const double* put, int aggressor, bool allin) {
        if (street == 2) return showdown(put);
        if (allin) return runout(street, put);
        budget();
        uint32_t id = add(kChance, 0, (uint8_t)(street + 1), put);
        std::vector<uint32_t> kids(52, kSentinel);
        for (int card = 0; card < 52; card++) {
            if ((bm_ >> card) & 1) continue;
            St n{street + 1, 0, {put[0], put[1]}, {0.0, 0.0}, 0.0, 0, aggressor, false};
            kids[card] = decision(n);
        }
        close_chance(id, kids);
        return id;
    }
    // tree.rs:725-759
    uint32_t runout(int street, const double* put) {
        budget();
        uint32_t id = add(kChance, 0, (uint8_t)(street + 1), put);
        std::vector<uint32_t> kids(52, kSentinel);
        for (int card = 0; card < 52; card++) {
            if ((bm_ >> card) & 1) continue;
            kids[card] = street + 1 == 2 ? showdown(put) : runout(street + 1, put);
        }
        close_chance(id, kids);
        return id;
    }
    void close_chance(uint32_t id, const std::vector<uint32_t>& kids) {
        t_.child_start[id] = (uint32_t)t_.children.size();
        t_.children.insert(t_.children.end(), kids.begin(), kids.end());
        t_.nchild[id] = 52;
    }
    // tree.rs:761-778
    uint32_t showdown(const double* put) {
        double rk = rake(put[0] + put[1]);
        uint32_t id = add(kShowdown, 0, 2, put);
        t_.twin[id] = put[0] - rk;
        t_.tlose[id] = -put[0];
        t_.ttie[id] = -rk / 2.0;
        return id;
    }
};
}  // namespace

// tree.rs:287-402
Tree build_tree(const TreeConfig& cfg, const std::vector<uint8_t>& board, uint64_t nh0, uint64_t nh1,
                uint64_t max_nodes, bool lenient) {
    if (board.size() < 3 || board.size() > 5) throw Error("board must have 3 to 5 cards");
    if (!(cfg.starting_pot > 0.0 && std::isfinite(cfg.starting_pot)) ||
        !(cfg.effective_stack > 0.0 && std::isfinite(cfg.effective_stack)))
        throw Error("pot and stacks must be positive finite numbers");
    const int rs = (int)board.size() - 3;
    static const char* kStreet[3] = {"flop", "turn", "river"};
    for (int p = 0; p < 2; p++)
        for (int s = 0; s < 3; s++) {
            const StreetSizing& z = cfg.side(p, s);
            for (const auto* l : {&z.bet, &z.raise, &z.donk})
                for (const BetSize& b : *l)
                    if (b.kind != kAllIn && !std::isfinite(b.v))
                        throw Error(std::string(kStreet[s]) + (p ? " IP" : " OOP") + ": size is not a finite number");
        }
    if (!lenient)
        for (int p = 0; p < 2; p++)
            for (int s = rs; s < 3; s++) {
                const StreetSizing& z = cfg.side(p, s);
                for (const BetSize& b : z.bet)
                    if (b.kind == kPrevMult)
                        throw Error(std::string(kStreet[s]) + (p ? " IP" : " OOP") +
                                    " bet: a raise multiple is a raise-only size; use % of pot or 'a'");
                if (p == 0 && s > rs)
                    for (const BetSize& b : z.donk)
                        if (b.kind == kPrevMult)
                            throw Error(std::string(kStreet[s]) +
                                        " OOP donk: a raise multiple is a raise-only size; use % of pot or 'a'");
            }
    uint64_t bm = 0;
    for (uint8_t c : board) bm |= 1ull << c;
    Builder b(cfg, rs, bm, max_nodes, nh0, nh1);
    double half = cfg.starting_pot / 2.0;
    St root{rs, 0, {half, half}, {0.0, 0.0}, 0.0, 0, -1, false};
    b.decision(root);
    return b.take();
}

// --------------------------------------------------------------------- spot
size_t Spot::river_key(const uint8_t* d, int n) const {  // game.rs:44-57
    if (tree.root_street == 2) return 0;
    if (tree.root_street == 1) return d[0];
    (void)n;
    return (size_t)std::min(d[0], d[1]) * 52 + std::max(d[0], d[1]);
}
const RiverBoard& Spot::river_at(const uint8_t* d, int n) const {
    const auto& e = river.at(river_key(d, n));
    if (!e) throw Error("river eval missing");
    return *e;
}
std::vector<int> Spot::perms_fixing(const uint8_t* d, int n) const {  // game.rs:335-344
    std::vector<int> out;
    for (size_t k = 0; k < perms.size(); k++) {
        bool ok = true;
        for (int i = 0; i < n; i++) ok = ok && card_permute(d[i], perms[k]) == d[i];
        if (ok) out.push_back((int)k);
    }
    return out;
}
size_t Spot::num_action_nodes() const {
    size_t c = 0;
    for (uint8_t k : tree.kind) c += k == kAction;
    return c;
}
double Spot::pair_weight_sum() const {  // best_response.rs:227-251
    double t = 0, s[52] = {0};
    for (size_t j = 0; j < hands[1].size(); j++) {
        double r = hands[1].w[j];
        t += r;
        s[hands[1].c1[j]] += r;
        s[hands[1].c2[j]] += r;
    }
    double total = 0;
    for (size_t i = 0; i < hands[0].size(); i++) {
        double same_r = same[0][i] != kSentinel ? (double)hands[1].w[same[0][i]] : 0.0;
        total += (double)hands[0].w[i] * (t - s[hands[0].c1[i]] - s[hands[0].c2[i]] + same_r);
    }
    return total;
}

static std::unique_ptr<RiverBoard> make_river_board(const Spot& sp, const uint8_t* extra, int ne) {  // game.rs:387-413
    auto rb = std::make_unique<RiverBoard>();
    uint8_t c7[7];
    size_t nb = sp.board.size();
    for (size_t i = 0; i < nb; i++) c7[i] = sp.board[i];
    uint64_t em = 0;
    for (int i = 0; i < ne; i++) { c7[nb + i] = extra[i]; em |= 1ull << extra[i]; }
    for (int p = 0; p < 2; p++) {
        const Hands& h = sp.hands[p];
        std::vector<uint64_t> keyed;  // strength << 16 | index sorts like (strength, index)
        keyed.reserve(h.size());
        for (size_t i = 0; i < h.size(); i++) {
            if (h.mask[i] & em) continue;
            c7[5] = h.c1[i];
            c7[6] = h.c2[i];
            keyed.push_back(((uint64_t)eval7(c7) << 16) | i);
        }
        std::sort(keyed.begin(), keyed.end());
        rb->str[p].resize(keyed.size());
        rb->idx[p].resize(keyed.size());
        for (size_t k = 0; k < keyed.size(); k++) {
            rb->str[p][k] = (uint32_t)(keyed[k] >> 16);
            rb->idx[p][k] = (uint16_t)(keyed[k] & 0xFFFF);
        }
    }
    return rb;
}

// game.rs:135-331
std::unique_ptr<Spot> build_spot(const SpotConfig& cfg, uint64_t max_nodes, bool lenient) {
    const TreeConfig& tc = cfg.tree;
    if (tc.rake_pct >= 1.0)
        throw Error("rake_pct is a FRACTION of the pot (0.05 = 5%), got a value >= 1 -- did you pass a percent?");
    if (tc.rake_pct < 0.0) throw Error("rake_pct must be >= 0");
    if (tc.rake_cap < 0.0) throw Error("rake_cap must be >= 0");
    auto sp = std::make_unique<Spot>();
    sp->config = cfg;
    sp->board = parse_board(cfg.board);
    if (sp->board.size() < 3 || sp->board.size() > 5) throw Error("board must have 3 to 5 cards");
    for (uint8_t c : sp->board) sp->board_mask |= 1ull << c;
    const std::string* rtext[2] = {&cfg.range_oop, &cfg.range_ip};
    for (int p = 0; p < 2; p++) {
        std::vector<float> w = parse_range_weights(*rtext[p]);
        Hands& h = sp->hands[p];
        for (int id = 0; id < 1326; id++) {
            if (!(w[id] > 0.0f)) continue;
            uint8_t hi, lo;
            combo_cards(id, &hi, &lo);
            uint64_t m = (1ull << hi) | (1ull << lo);
            if (m & sp->board_mask) continue;
            h.c1.push_back(hi);
            h.c2.push_back(lo);
            h.w.push_back(w[id]);
            h.mask.push_back(m);
        }
        if (h.size() == 0)
            throw Error(std::string(p == 0 ? "OOP" : "IP") + " range has no combos left after board card removal");
        if (h.size() > 65535) throw Error("range too large");
    }
    double mass = 0;
    for (size_t i = 0; i < sp->hands[0].size(); i++)
        for (size_t j = 0; j < sp->hands[1].size(); j++)
            if (!(sp->hands[0].mask[i] & sp->hands[1].mask[j])) mass += (double)sp->hands[0].w[i] * sp->hands[1].w[j];
    if (mass <= 0.0)
        throw Error("OOP and IP ranges are mutually impossible: every OOP combo shares a card with every IP combo");
    int pos_of[2][1326];
    for (int p = 0; p < 2; p++) {
        std::fill(pos_of[p], pos_of[p] + 1326, -1);
        for (size_t i = 0; i < sp->hands[p].size(); i++)
            pos_of[p][combo_id(sp->hands[p].c1[i], sp->hands[p].c2[i])] = (int)i;
    }
    for (int p = 0; p < 2; p++)
        for (size_t i = 0; i < sp->hands[p].size(); i++) {
            int j = pos_of[1 - p][combo_id(sp->hands[p].c1[i], sp->hands[p].c2[i])];
            sp->same[p].push_back(j < 0 ? kSentinel : (uint32_t)j);
        }
    sp->tree = build_tree(tc, sp->board, sp->hands[0].size(), sp->hands[1].size(), max_nodes, lenient);

    // river strength tables (game.rs:384-462), one per completed board
    const int rs = sp->tree.root_street;
    std::vector<std::vector<uint8_t>> extras;
    if (rs == 2) {
        sp->river.resize(1);
        extras.push_back({});
    } else if (rs == 1) {
        sp->river.resize(52);
        for (int c = 0; c < 52; c++)
            if (!((sp->board_mask >> c) & 1)) extras.push_back({(uint8_t)c});
    } else {
        sp->river.resize(52 * 52);
        for (int a = 0; a < 52; a++)
            for (int b = a + 1; b < 52; b++)
                if (!((sp->board_mask >> a) & 1) && !((sp->board_mask >> b) & 1)) extras.push_back({(uint8_t)a, (uint8_t)b});
    }
    {
        unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; t++)
            pool.emplace_back([&, t]() {
                for (size_t k = t; k < extras.size(); k += nt) {
                    const auto& e = extras[k];
                    auto rb = make_river_board(*sp, e.data(), (int)e.size());
                    sp->river[sp->river_key(e.data(), (int)e.size())] = std::move(rb);
                }
            });
        for (auto& th : pool) th.join();
    }

    // suit symmetries fixing the board pointwise and both ranges (game.rs:260-317)
    std::array<uint8_t, 4> pm;
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++)
            for (int c = 0; c < 4; c++)
                for (int d = 0; d < 4; d++) {
                    if (a == b || a == c || a == d || b == c || b == d || c == d) continue;
                    pm = {(uint8_t)a, (uint8_t)b, (uint8_t)c, (uint8_t)d};
                    bool ok = true;
                    for (uint8_t x : sp->board) ok = ok && card_permute(x, pm) == x;
                    std::vector<uint16_t> tb[2];
                    for (int p = 0; p < 2 && ok; p++) {
                        const Hands& h = sp->hands[p];
                        for (size_t i = 0; i < h.size() && ok; i++) {
                            int j = pos_of[p][combo_id(card_permute(h.c1[i], pm), card_permute(h.c2[i], pm))];
                            ok = j >= 0 && std::fabs(h.w[j] - h.w[i]) < 1e-6f;
                            if (ok) tb[p].push_back((uint16_t)j);
                        }
                    }
                    if (!ok) continue;
                    sp->perms.push_back(pm);
                    sp->hand_perm[0].push_back(std::move(tb[0]));
                    sp->hand_perm[1].push_back(std::move(tb[1]));
                }
    for (size_t k = 0; k < sp->perms.size(); k++)
        if (sp->perms[k] == std::array<uint8_t, 4>{0, 1, 2, 3}) {
            std::swap(sp->perms[0], sp->perms[k]);
            std::swap(sp->hand_perm[0][0], sp->hand_perm[0][k]);
            std::swap(sp->hand_perm[1][0], sp->hand_perm[1][k]);
            break;
        }
    return sp;
}

}  // namespace gtob
