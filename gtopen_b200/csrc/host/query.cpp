#include "query.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <limits>

#include "../kernels/engine.hpp"
#include "batch.hpp"

namespace gtob {

namespace {
// Hand index of (hi, lo) for player p, -1 if not in the range.
std::vector<int> combo_index(const Spot& sp, int p) {
    std::vector<int> ix(52 * 52, -1);
    const Hands& h = sp.hands[p];
    for (size_t i = 0; i < h.size(); i++) ix[h.c1[i] * 52 + h.c2[i]] = (int)i;
    return ix;
}
// For each hand of p, the index of its image under the suit permutation.
std::vector<int> hand_map(const Spot& sp, int p, const std::array<uint8_t, 4>& perm) {
    const std::vector<int> ix = combo_index(sp, p);
    const Hands& h = sp.hands[p];
    std::vector<int> m(h.size());
    for (size_t i = 0; i < h.size(); i++) {
        uint8_t a = card_permute(h.c1[i], perm), b = card_permute(h.c2[i], perm);
        if (a < b) std::swap(a, b);
        m[i] = ix[a * 52 + b];
        if (m[i] < 0) throw Error("suit permutation maps a hand outside the range");
    }
    return m;
}
// fold_cfv of game.rs:470-496 (f64 totals, f32 result).
void fold_values(const Spot& sp, int p, const float* ro, float amount, float* out) {
    const Hands& ho = sp.hands[1 - p];
    double t = 0.0, s[52] = {0.0};
    for (size_t j = 0; j < ho.size(); j++) {
        t += (double)ro[j];
        s[ho.c1[j]] += (double)ro[j];
        s[ho.c2[j]] += (double)ro[j];
    }
    const Hands& hp = sp.hands[p];
    for (size_t i = 0; i < hp.size(); i++) {
        const uint32_t same = sp.same[p][i];
        const float same_r = same != kSentinel ? ro[same] : 0.0f;
        out[i] = amount * ((float)(t - s[hp.c1[i]] - s[hp.c2[i]]) + same_r);
    }
}
// sweep_buckets (game.rs:580-653): win / tie / valid opponent mass of each
// of p's hands on one complete board.
void sweep_buckets(const RiverBoard& rb, const Spot& sp, int p, const float* ro, double* win, double* tie,
                   double* valid) {
    const std::vector<uint32_t>& ms = rb.str[p];
    const std::vector<uint16_t>& mi = rb.idx[p];
    const std::vector<uint32_t>& os = rb.str[1 - p];
    const std::vector<uint16_t>& oi = rb.idx[1 - p];
    const Hands& hm = sp.hands[p];
    const Hands& ho = sp.hands[1 - p];
    double t_all = 0.0, s_all[52] = {0.0};
    for (size_t j = 0; j < oi.size(); j++) {
        const double r = (double)ro[oi[j]];
        t_all += r;
        s_all[ho.c1[oi[j]]] += r;
        s_all[ho.c2[oi[j]]] += r;
    }
    std::vector<double> lower(mi.size());
    {
        double t = 0.0, s[52] = {0.0};
        size_t j = 0;
        for (size_t k = 0; k < mi.size(); k++) {
            while (j < oi.size() && os[j] < ms[k]) {
                const double r = (double)ro[oi[j]];
                t += r;
                s[ho.c1[oi[j]]] += r;
                s[ho.c2[oi[j]]] += r;
                j++;
            }
            lower[k] = t - s[hm.c1[mi[k]]] - s[hm.c2[mi[k]]];
        }
    }
    double t = 0.0, s[52] = {0.0};
    size_t j = oi.size();
    for (size_t k = mi.size(); k-- > 0;) {
        while (j > 0 && os[j - 1] > ms[k]) {
            j--;
            const double r = (double)ro[oi[j]];
            t += r;
            s[ho.c1[oi[j]]] += r;
            s[ho.c2[oi[j]]] += r;
        }
        const int i = mi[k];
        const double higher = t - s[hm.c1[i]] - s[hm.c2[i]];
        const uint32_t same = sp.same[p][i];
        const double same_r = same != kSentinel ? (double)ro[same] : 0.0;
        const double v = t_all - s_all[hm.c1[i]] - s_all[hm.c2[i]] + same_r;
        win[i] += lower[k];
        tie[i] += v - lower[k] - higher;
        valid[i] += v;
    }
}
}  // namespace

std::vector<float> equity(const Spot& sp, int p, const float* reach_o, const uint8_t* dealt, int nd) {
    const size_t nh = sp.hands[p].size(), no = sp.hands[1 - p].size();
    std::vector<double> win(nh, 0.0), tie(nh, 0.0), valid(nh, 0.0);
    const Hands& ho = sp.hands[1 - p];
    auto blocked = [&](int c) {
        if (sp.board_mask >> c & 1) return true;
        for (int i = 0; i < nd; i++)
            if (dealt[i] == c) return true;
        return false;
    };
    const int board_len = (int)sp.board.size() + nd;
    if (board_len == 5) {
        sweep_buckets(sp.river_at(dealt, nd), sp, p, reach_o, win.data(), tie.data(), valid.data());
    } else if (board_len == 4) {
        std::vector<float> ro(no);
        uint8_t d2[2] = {nd > 0 ? dealt[0] : (uint8_t)0, 0};
        for (int c = 0; c < 52; c++) {
            if (blocked(c)) continue;
            for (size_t j = 0; j < no; j++) ro[j] = (ho.mask[j] >> c & 1) ? 0.0f : reach_o[j];
            d2[nd] = (uint8_t)c;
            sweep_buckets(sp.river_at(d2, nd + 1), sp, p, ro.data(), win.data(), tie.data(), valid.data());
        }
    } else {
        std::vector<float> rt(no), ro(no);
        for (int tc = 0; tc < 52; tc++) {
            if (sp.board_mask >> tc & 1) continue;
            for (size_t j = 0; j < no; j++) rt[j] = (ho.mask[j] >> tc & 1) ? 0.0f : reach_o[j];
            for (int rc = tc + 1; rc < 52; rc++) {
                if (sp.board_mask >> rc & 1) continue;
                for (size_t j = 0; j < no; j++) ro[j] = (ho.mask[j] >> rc & 1) ? 0.0f : rt[j];
                const uint8_t d2[2] = {(uint8_t)tc, (uint8_t)rc};
                sweep_buckets(sp.river_at(d2, 2), sp, p, ro.data(), win.data(), tie.data(), valid.data());
            }
        }
    }
    std::vector<float> out(nh);
    for (size_t i = 0; i < nh; i++)
        out[i] = valid[i] > 1e-12 ? (float)((win[i] + 0.5 * tie[i]) / valid[i]) : std::numeric_limits<float>::quiet_NaN();
    return out;
}

// walk_path (query.rs:304-340) with each action node's strategy from the
// device block of its representative under the prefix's suit permutation.
static uint32_t walk_device(GpuEngine& eng, const HostSolver& host, const std::vector<int>& steps,
                            std::vector<float> reach[2]) {
    const Spot& sp = *host.spot;
    const Tree& t = sp.tree;
    reach[0] = sp.hands[0].w;
    reach[1] = sp.hands[1].w;
    uint32_t n = 0;
    uint8_t dealt[2];
    int nd = 0;
    for (size_t k = 0; k < steps.size(); k++) {
        const int s = steps[k];
        if (t.kind[n] == kAction && s >= 0) {
            const int na = t.nchild[n], p = t.player[n];
            if (s >= na) throw Error("action index " + std::to_string(s) + " out of range");
            const size_t nh = sp.hands[p].size();
            std::array<uint8_t, 4> perm;
            const std::vector<int> prefix(steps.begin(), steps.begin() + k);
            uint32_t cn;
            std::vector<float> unused[2];
            host.walk(host.canonical_steps(prefix, &perm), &cn, unused);
            std::vector<float> sig(na * nh);
            auto lk = host.locks.find(cn);
            if (lk != host.locks.end()) sig = lk->second;
            else eng.node_average_strategy(cn, sig.data());
            const std::vector<int> m = hand_map(sp, p, perm);
            for (size_t i = 0; i < nh; i++) reach[p][i] *= sig[s * nh + m[i]];
            n = t.child(n, s);
        } else if (t.kind[n] == kChance && s < 0) {
            const uint8_t c = (uint8_t)(-1 - s);
            bool was = false;
            for (int i = 0; i < nd; i++) was = was || dealt[i] == c;
            const uint32_t ch = t.children[t.child_start[n] + c];
            if (ch == kSentinel || was) throw Error("card " + card_name(c) + " not available here");
            for (int p = 0; p < 2; p++)
                for (size_t i = 0; i < sp.hands[p].size(); i++)
                    if (sp.hands[p].mask[i] >> c & 1) reach[p][i] = 0.0f;
            if (nd < 2) dealt[nd++] = c;
            n = ch;
        } else {
            throw Error("path step does not match the node kind");
        }
    }
    return n;
}

// The cards a path deals, in order.
static int path_dealt(const std::vector<int>& steps, uint8_t* dealt) {
    int nd = 0;
    for (int s : steps)
        if (s < 0 && nd < 2) dealt[nd++] = (uint8_t)(-1 - s);
    return nd;
}

NodeValues node_values(GpuEngine& eng, const HostSolver& host, const std::vector<int>& steps) {
    const Spot& sp = *host.spot;
    const Tree& t = sp.tree;
    const float nan = std::numeric_limits<float>::quiet_NaN();
    NodeValues out;
    const uint32_t n = walk_device(eng, host, steps, out.reach);
    uint8_t dealt[2];
    const int nd = path_dealt(steps, dealt);
    for (int p = 0; p < 2; p++) out.eq[p] = equity(sp, p, out.reach[1 - p].data(), dealt, nd);
    out.node = n;
    out.kind = t.kind[n];
    out.player = t.kind[n] == kAction ? t.player[n] : -1;
    out.na = t.kind[n] == kAction ? t.nchild[n] : 0;
    // the representative the device holds, and the hand maps onto it
    std::array<uint8_t, 4> perm;
    const std::vector<int> canon = host.canonical_steps(steps, &perm);
    uint32_t cn;
    std::vector<float> unused[2];
    host.walk(canon, &cn, unused);
    // a fold terminal has no slot: its values come from the walk reach; any
    // other node is read from the sweep (an in-place showdown, under the fused
    // engine, from its parent's -- not supported: the staged engine's have slots)
    const bool fold_end = t.kind[n] == kFold;
    for (int p = 0; p < 2; p++) {
        const int nh = (int)sp.hands[p].size();
        const float* ro = out.reach[1 - p].data();
        const std::vector<double> valid = valid_opp_sum(sp, p, ro);
        out.valid[p].resize(nh);
        for (int i = 0; i < nh; i++) out.valid[p][i] = (float)valid[i];
        const double put = p == 0 ? t.put0[n] : t.put1[n];
        const std::vector<int> m = hand_map(sp, p, perm);
        std::vector<float> cfv(nh, 0.0f), cfv_c(nh, 0.0f);
        const bool actor = t.kind[n] == kAction && t.player[n] == p;
        const int na = actor ? t.nchild[n] : 0;
        std::vector<float> child_c((size_t)na * nh, 0.0f);
        std::vector<uint8_t> ok(na, 0);
        if (fold_end) {
            fold_values(sp, p, ro, (float)(t.player[n] == p ? t.tlose[n] : t.twin[n]), cfv.data());
        } else {
            eng.node_sweep_values(cn, p, 1, cfv_c.data(), nullptr, nullptr, actor ? child_c.data() : nullptr, ok.data());
            for (int i = 0; i < nh; i++) cfv[i] = cfv_c[m[i]];
        }
        out.ev[p].assign(nh, nan);
        if (!actor) {
            for (int i = 0; i < nh; i++)
                if (valid[i] > 1e-9) out.ev[p][i] = (float)((double)cfv[i] / valid[i] + put);
            continue;
        }
        // the actor: average strategy, one EV per action (query.rs:530-556)
        out.strategy.assign((size_t)na * nh, 0.0f);
        {
            std::vector<float> sig((size_t)na * nh);
            auto lk = host.locks.find(cn);
            if (lk != host.locks.end()) sig = lk->second;
            else eng.node_average_strategy(cn, sig.data());
            for (int a = 0; a < na; a++)
                for (int i = 0; i < nh; i++) out.strategy[(size_t)a * nh + i] = sig[(size_t)a * nh + m[i]];
        }
        out.action_ev.assign((size_t)na * nh, nan);
        std::vector<double> total(nh, 0.0);
        std::vector<float> cv(nh);
        for (int a = 0; a < na; a++) {
            const uint32_t c = t.child(n, a);
            if (ok[a]) {
                for (int i = 0; i < nh; i++) cv[i] = child_c[(size_t)a * nh + m[i]];
            } else {  // a fold child evaluated in place: from the walk reach
                if (t.kind[c] != kFold) throw Error("node values need the staged or plain engine (showdowns with slots)");
                fold_values(sp, p, ro, (float)(t.player[c] == p ? t.tlose[c] : t.twin[c]), cv.data());
            }
            for (int i = 0; i < nh; i++)
                if (valid[i] > 1e-9) {
                    const double ev = (double)cv[i] / valid[i] + put;
                    out.action_ev[(size_t)a * nh + i] = (float)ev;
                    total[i] += (double)out.strategy[(size_t)a * nh + i] * ev;
                }
        }
        for (int i = 0; i < nh; i++)
            if (valid[i] > 1e-9) out.ev[p][i] = (float)total[i];
    }
    return out;
}

Runouts runouts(GpuEngine& eng, const HostSolver& host, const std::vector<int>& steps) {
    const Spot& sp = *host.spot;
    const Tree& t = sp.tree;
    const float nan = std::numeric_limits<float>::quiet_NaN();
    std::vector<float> reach[2];
    const uint32_t n = walk_device(eng, host, steps, reach);
    if (t.kind[n] != kChance) throw Error("runouts report requires a chance (card) node");
    uint8_t dealt[2];
    const int nd = path_dealt(steps, dealt);
    Runouts out;
    struct Card {
        int c;
        uint32_t child, canon;
        std::array<uint8_t, 4> perm;
    };
    std::vector<Card> cards;
    for (int c = 51; c >= 0; c--) {
        const uint32_t ch = t.children[t.child_start[n] + c];
        bool was = false;
        for (int i = 0; i < nd; i++) was = was || dealt[i] == c;
        if (ch == kSentinel || was) continue;
        std::vector<int> st = steps;
        st.push_back(-1 - c);
        Card e{c, ch, 0, {0, 1, 2, 3}};
        std::vector<float> unused[2];
        host.walk(host.canonical_steps(st, &e.perm), &e.canon, unused);
        cards.push_back(e);
    }
    // the children's average-strategy values, one sweep per player
    std::vector<uint32_t> uniq;
    for (auto& e : cards)
        if (std::find(uniq.begin(), uniq.end(), e.canon) == uniq.end()) uniq.push_back(e.canon);
    std::vector<float> vals[2];
    std::vector<uint8_t> ok[2];
    for (int p = 0; p < 2; p++) {
        vals[p].assign(uniq.size() * sp.hands[p].size(), 0.0f);
        ok[p].assign(uniq.size(), 0);
        eng.sweep_values(p, 1, uniq.data(), (int)uniq.size(), vals[p].data(), ok[p].data());
    }
    for (auto& e : cards) {
        const uint32_t ch = e.child;
        RunoutRow row;
        row.card = e.c;
        std::vector<float> rc[2] = {reach[0], reach[1]};
        for (int p = 0; p < 2; p++)
            for (size_t i = 0; i < rc[p].size(); i++)
                if (sp.hands[p].mask[i] >> e.c & 1) rc[p][i] = 0.0f;
        if (t.kind[ch] == kAction) {
            const int p = t.player[ch], na = t.nchild[ch];
            const size_t nh = sp.hands[p].size();
            out.player = p;
            out.na = na;
            std::vector<float> sig((size_t)na * nh);
            auto lk = host.locks.find(e.canon);
            if (lk != host.locks.end()) sig = lk->second;
            else eng.node_average_strategy(e.canon, sig.data());
            const std::vector<int> m = hand_map(sp, p, e.perm);
            double total = 0.0;
            std::vector<double> sums(na, 0.0);
            for (size_t i = 0; i < nh; i++) {
                const double r = (double)rc[p][i];
                total += r;
                for (int a = 0; a < na; a++) sums[a] += r * (double)sig[(size_t)a * nh + m[i]];
            }
            for (int a = 0; a < na; a++) row.freqs.push_back(total > 1e-12 ? (float)(sums[a] / total) : 0.0f);
        }
        uint8_t d2[2] = {nd > 0 ? dealt[0] : (uint8_t)0, 0};
        d2[nd] = (uint8_t)e.c;
        const size_t u = (size_t)(std::find(uniq.begin(), uniq.end(), e.canon) - uniq.begin());
        for (int p = 0; p < 2; p++) {
            const size_t nh = sp.hands[p].size();
            const float* ro = rc[1 - p].data();
            const std::vector<double> valid = valid_opp_sum(sp, p, ro);
            const std::vector<float> eq = equity(sp, p, ro, d2, nd + 1);
            double num = 0.0, den = 0.0;
            for (size_t i = 0; i < nh; i++)
                if (!std::isnan(eq[i])) {
                    const double w = (double)rc[p][i] * valid[i];
                    num += w * (double)eq[i];
                    den += w;
                }
            row.eq[p] = den > 1e-12 ? (float)(num / den) : nan;
            std::vector<float> cfv(nh, 0.0f);
            if (ok[p][u]) {
                const std::vector<int> m = hand_map(sp, p, e.perm);
                for (size_t i = 0; i < nh; i++) cfv[i] = vals[p][u * nh + m[i]];
            } else if (t.kind[ch] == kFold) {
                fold_values(sp, p, ro, (float)(t.player[ch] == p ? t.tlose[ch] : t.twin[ch]), cfv.data());
            } else {
                throw Error("runouts need the staged or plain engine (showdowns with slots)");
            }
            const double put = p == 0 ? t.put0[ch] : t.put1[ch];
            num = den = 0.0;
            for (size_t i = 0; i < nh; i++)
                if (valid[i] > 1e-9 && rc[p][i] > 0.0f) {
                    const double w = (double)rc[p][i] * valid[i];
                    num += w * ((double)cfv[i] / valid[i] + put);
                    den += w;
                }
            row.ev[p] = den > 1e-12 ? (float)(num / den) : nan;
        }
        if (out.pot == 0.0) out.pot = t.put0[ch] + t.put1[ch];
        out.rows.push_back(std::move(row));
    }
    return out;
}

ExploitValues exploit_values(GpuEngine& eng, const HostSolver& host, const std::vector<int>& steps, int p) {
    if (p != 0 && p != 1) throw Error("exploiter must be 0 (OOP) or 1 (IP)");
    const Spot& sp = *host.spot;
    const Tree& t = sp.tree;
    const float nan = std::numeric_limits<float>::quiet_NaN();
    ExploitValues out;
    std::array<uint8_t, 4> perm;
    const std::vector<int> canon = host.canonical_steps(steps, &perm);
    std::vector<float> reach[2];
    const uint32_t n = walk_device(eng, host, canon, reach);  // query.rs:815: the canonical walk
    out.node = n;
    out.kind = t.kind[n];
    out.player = t.kind[n] == kAction ? t.player[n] : -1;
    const int nh = (int)sp.hands[p].size();
    const float* ro = reach[1 - p].data();
    const std::vector<double> valid = valid_opp_sum(sp, p, ro);
    const std::vector<int> tbl = hand_map(sp, p, perm);
    const bool actor = t.kind[n] == kAction && t.player[n] == p;
    const int na = t.kind[n] == kAction ? t.nchild[n] : 0;
    out.na = na;
    auto lk = host.locks.find(n);
    const std::vector<float>* lock = lk != host.locks.end() ? &lk->second : nullptr;
    const double put = p == 0 ? t.put0[n] : t.put1[n];
    const bool fold_end = t.kind[n] == kFold;
    const float famount = fold_end ? (float)(t.player[n] == p ? t.tlose[n] : t.twin[n]) : 0.0f;
    // best-response values: per action where p acts, else the node's
    std::vector<float> acfv((size_t)na * nh, 0.0f), br(nh, 0.0f), cur(nh, 0.0f);
    std::vector<uint8_t> ok(na, 0);
    if (fold_end) {
        fold_values(sp, p, ro, famount, br.data());
        cur = br;
    } else {
        eng.node_sweep_values(n, p, 0, actor ? nullptr : br.data(), nullptr, nullptr, actor ? acfv.data() : nullptr,
                              ok.data());
        eng.node_sweep_values(n, p, 1, cur.data(), nullptr, nullptr, nullptr, nullptr);
    }
    if (actor) {
        for (int a = 0; a < na; a++)
            if (!ok[a]) {
                const uint32_t c = t.child(n, a);
                if (t.kind[c] != kFold) throw Error("exploit values need the staged or plain engine (showdowns with slots)");
                fold_values(sp, p, ro, (float)(t.player[c] == p ? t.tlose[c] : t.twin[c]), acfv.data() + (size_t)a * nh);
            }
        for (int i = 0; i < nh; i++) {
            if (lock) {
                float v = 0.0f;
                for (int a = 0; a < na; a++) v += (*lock)[(size_t)a * nh + i] * acfv[(size_t)a * nh + i];
                br[i] = v;
            } else {
                float v = -std::numeric_limits<float>::infinity();
                for (int a = 0; a < na; a++) v = std::fmax(v, acfv[(size_t)a * nh + i]);
                br[i] = v;
            }
        }
    }
    auto ev_of = [&](float cfv, int j) { return valid[j] > 1e-9 ? (float)((double)cfv / valid[j] + put) : nan; };
    out.reach.resize(nh);
    out.valid.resize(nh);
    out.br_ev.resize(nh);
    out.cur_ev.resize(nh);
    out.gain.resize(nh);
    if (actor) {
        out.br_strategy.assign((size_t)na * nh, 0.0f);
        out.action_ev.assign((size_t)na * nh, nan);
    }
    double wsum = 0.0, bs = 0.0, cs = 0.0;
    for (int i = 0; i < nh; i++) {
        const int j = tbl[i];
        out.reach[i] = reach[p][j];
        out.valid[i] = (float)valid[j];
        const float b = ev_of(br[j], j), c = ev_of(cur[j], j);
        out.br_ev[i] = b;
        out.cur_ev[i] = c;
        out.gain[i] = (!std::isnan(b) && !std::isnan(c)) ? b - c : nan;
        if (actor) {
            if (lock) {
                for (int a = 0; a < na; a++) out.br_strategy[(size_t)a * nh + i] = (*lock)[(size_t)a * nh + j];
            } else {
                float m = -std::numeric_limits<float>::infinity();
                for (int a = 0; a < na; a++) m = std::fmax(m, acfv[(size_t)a * nh + j]);
                const float eps = std::fmax(std::fabs(m) * 1e-5f, 1e-5f);
                int w = 0;
                for (int a = 0; a < na; a++) w += (m - acfv[(size_t)a * nh + j] <= eps) ? 1 : 0;
                const float wf = (float)std::max(w, 1);
                for (int a = 0; a < na; a++)
                    out.br_strategy[(size_t)a * nh + i] = (m - acfv[(size_t)a * nh + j] <= eps) ? 1.0f / wf : 0.0f;
            }
            for (int a = 0; a < na; a++) out.action_ev[(size_t)a * nh + i] = ev_of(acfv[(size_t)a * nh + j], j);
        }
        if (!std::isnan(b) && !std::isnan(c)) {  // query.rs:901-913
            const double w = (double)out.reach[i] * (double)out.valid[i];
            if (w > 0.0) {
                wsum += w;
                bs += w * (double)b;
                cs += w * (double)c;
            }
        }
    }
    if (wsum > 1e-12) {
        out.avg[0] = (float)(bs / wsum);
        out.avg[1] = (float)(cs / wsum);
        out.avg[2] = (float)((bs - cs) / wsum);
    } else {
        out.avg[0] = out.avg[1] = out.avg[2] = nan;
    }
    return out;
}

// ------------------------------------------------ node_view's structure
namespace {
// tree.rs:163-169: an integral amount as an integer, else two decimals
std::string trim_num(double x) {
    if (std::fabs(x - std::round(x)) < 1e-6) return std::to_string((long long)std::round(x));
    char b[64];
    std::snprintf(b, sizeof(b), "%.2f", x);
    return b;
}
// an integral f64 printed as Rust's `{}` prints it (the bet label's percentage)
std::string rust_int_f64(double x) {
    if (x == 0.0) return std::signbit(x) ? "-0" : "0";
    char b[64];
    std::snprintf(b, sizeof(b), "%.0f", x);
    return b;
}
const char* act_kind_name(int k) {
    switch (k) {
        case kFoldA: return "fold";
        case kCheck: return "check";
        case kCall: return "call";
        case kBet: return "bet";
        default: return "raise";
    }
}
// query.rs:353-394 action_views
json::Value action_views(const Spot& sp, uint32_t n) {
    const Tree& t = sp.tree;
    json::Value arr = json::Value::array();
    if (t.kind[n] != kAction) return arr;
    const double pot = t.put0[n] + t.put1[n];
    const int me = t.player[n];
    const TreeConfig& cfg = sp.config.tree;
    for (int a = 0; a < t.nchild[n]; a++) {
        const int k = t.act_kind[t.action_start[n] + a];
        const double amt = t.act_amount[t.action_start[n] + a];
        bool all_in = false;
        if (k == kBet || k == kRaise) {
            const uint32_t c = t.child(n, a);
            const double put = me == 0 ? t.put0[c] : t.put1[c];
            all_in = std::fabs(cfg.effective_stack - (put - cfg.starting_pot / 2.0)) < 1e-6;
        }
        std::string label;
        switch (k) {
            case kFoldA: label = "Fold"; break;
            case kCheck: label = "Check"; break;
            case kCall: label = "Call"; break;
            case kBet:
                label = all_in ? "All-in " + trim_num(amt)
                               : "Bet " + trim_num(amt) + " (" + rust_int_f64(std::round(amt / pot * 100.0)) + "%)";
                break;
            default: label = all_in ? "All-in " + trim_num(amt) : "Raise " + trim_num(amt); break;
        }
        json::Value v = json::Value::object();
        v.set("label", json::Value::string(label));
        v.set("kind", json::Value::string(act_kind_name(k)));
        v.set("amount", json::Value::number(k == kCall || k == kBet || k == kRaise ? amt : 0.0));
        arr.arr.push_back(std::move(v));
    }
    return arr;
}
json::Value opt_int(bool has, long long v) { return has ? json::Value::integer(v) : json::Value(); }
}  // namespace

std::string path_view_json(const HostSolver& host, const std::vector<int>& steps) {
    const Spot& sp = *host.spot;
    const Tree& t = sp.tree;
    const TreeConfig& cfg = sp.config.tree;
    auto stack_of = [&](uint32_t n) {
        const int p = t.player[n];
        return cfg.effective_stack - ((p == 0 ? t.put0[n] : t.put1[n]) - cfg.starting_pot / 2.0);
    };
    json::Value history = json::Value::array();
    std::vector<uint8_t> dealt;
    uint32_t n = 0;
    for (int st : steps) {  // query.rs:396-461 build_history, walk_path's checks
        json::Value h = json::Value::object();
        if (t.kind[n] == kAction && st >= 0) {
            if (st >= t.nchild[n]) throw Error("invalid argument: action index out of range");
            h.set("kind", json::Value::string("action"));
            h.set("player", json::Value::integer(t.player[n]));
            h.set("stack", json::Value::number(stack_of(n)));
            h.set("pot", json::Value::number(t.put0[n] + t.put1[n]));
            h.set("street", json::Value::integer(t.street[n]));
            h.set("actions", action_views(sp, n));
            h.set("chosen", json::Value::integer(st));
            h.set("card", json::Value());
            n = t.child(n, st);
        } else if (t.kind[n] == kChance && st < 0) {
            const int c = -1 - st;
            if (c >= 52 || t.child(n, c) == kSentinel || std::find(dealt.begin(), dealt.end(), (uint8_t)c) != dealt.end())
                throw Error("invalid argument: card " + std::to_string(c) + " cannot be dealt here");
            h.set("kind", json::Value::string("card"));
            h.set("player", json::Value());
            h.set("stack", json::Value::number(0.0));
            h.set("pot", json::Value::number(t.put0[n] + t.put1[n]));
            h.set("street", json::Value::integer(t.street[n]));
            h.set("actions", json::Value::array());
            h.set("chosen", json::Value());
            h.set("card", json::Value::string(card_name((uint8_t)c)));
            dealt.push_back((uint8_t)c);
            n = t.child(n, c);
        } else {
            throw Error("invalid argument: path step does not match node type");
        }
        history.arr.push_back(std::move(h));
    }
    const bool act = t.kind[n] == kAction;
    {
        json::Value h = json::Value::object();
        h.set("kind", json::Value::string(act ? "action" : t.kind[n] == kChance ? "card" : "terminal"));
        h.set("player", opt_int(act, t.player[n]));
        h.set("stack", json::Value::number(act ? stack_of(n) : 0.0));
        h.set("pot", json::Value::number(t.put0[n] + t.put1[n]));
        h.set("street", json::Value::integer(t.street[n]));
        h.set("actions", action_views(sp, n));
        h.set("chosen", json::Value());
        h.set("card", json::Value());
        history.arr.push_back(std::move(h));
    }
    static const char* kTypes[4] = {"action", "chance", "terminal_fold", "terminal_showdown"};
    json::Value v = json::Value::object();
    v.set("node", json::Value::integer(n));
    v.set("node_type", json::Value::string(t.kind[n] < 4 ? kTypes[t.kind[n]] : "?"));
    v.set("street", json::Value::integer(t.street[n]));
    json::Value board = json::Value::array();
    for (uint8_t c : sp.board) board.arr.push_back(json::Value::string(card_name(c)));
    for (uint8_t c : dealt) board.arr.push_back(json::Value::string(card_name(c)));
    v.set("board", board);
    v.set("pot", json::Value::number(t.put0[n] + t.put1[n]));
    json::Value put = json::Value::array();
    put.arr.push_back(json::Value::number(t.put0[n]));
    put.arr.push_back(json::Value::number(t.put1[n]));
    v.set("put", put);
    v.set("player", opt_int(act, t.player[n]));
    v.set("actions", action_views(sp, n));
    if (t.kind[n] == kChance) {
        json::Value cards = json::Value::array();
        for (int c = 0; c < 52; c++)
            if (t.child(n, c) != kSentinel && std::find(dealt.begin(), dealt.end(), (uint8_t)c) == dealt.end())
                cards.arr.push_back(json::Value::string(card_name((uint8_t)c)));
        v.set("available_cards", cards);
    } else {
        v.set("available_cards", json::Value());
    }
    // the lock lives on the orbit representative's node (query.rs:627-633)
    bool locked = false;
    {
        std::array<uint8_t, 4> perm;
        const std::vector<int> canon = host.canonical_steps(steps, &perm);
        uint32_t m = 0;
        for (int st : canon) m = st >= 0 ? t.child(m, st) : t.child(m, -1 - st);
        locked = host.locks.count(m) > 0;
    }
    v.set("locked", json::Value::boolean(locked));
    v.set("history", history);
    return json::dump(v);
}

}  // namespace gtob
