#include "query.hpp"

#include <cmath>
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
}  // namespace

NodeValues node_values(GpuEngine& eng, const HostSolver& host, const std::vector<int>& steps) {
    const Spot& sp = *host.spot;
    const Tree& t = sp.tree;
    const float nan = std::numeric_limits<float>::quiet_NaN();
    NodeValues out;
    // walk the path (query.rs:304-340), each action node's strategy from the
    // device block of its representative under the prefix's suit permutation
    out.reach[0] = sp.hands[0].w;
    out.reach[1] = sp.hands[1].w;
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
            for (size_t i = 0; i < nh; i++) out.reach[p][i] *= sig[s * nh + m[i]];
            n = t.child(n, s);
        } else if (t.kind[n] == kChance && s < 0) {
            const uint8_t c = (uint8_t)(-1 - s);
            bool was = false;
            for (int i = 0; i < nd; i++) was = was || dealt[i] == c;
            const uint32_t ch = t.children[t.child_start[n] + c];
            if (ch == kSentinel || was) throw Error("card " + card_name(c) + " not available here");
            for (int p = 0; p < 2; p++)
                for (size_t i = 0; i < sp.hands[p].size(); i++)
                    if (sp.hands[p].mask[i] >> c & 1) out.reach[p][i] = 0.0f;
            if (nd < 2) dealt[nd++] = c;
            n = ch;
        } else {
            throw Error("path step does not match the node kind");
        }
    }
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
            eng.node_sweep_values(cn, p, cfv_c.data(), nullptr, nullptr, actor ? child_c.data() : nullptr, ok.data());
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

}  // namespace gtob
