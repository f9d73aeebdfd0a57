// Host solver state, .gto save/load, locks and symmetrisation: see solver.hpp.
#include "solver.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sys/stat.h>
#include <unistd.h>

namespace gtob {

// ------------------------------------------------------------ store.rs codecs
static inline int16_t sat_i16(float x) {  // Rust `as i16`: saturating, NaN -> 0
    if (std::isnan(x)) return 0;
    return x >= 32767.0f ? 32767 : x <= -32768.0f ? -32768 : (int16_t)x;
}
static inline uint16_t sat_u16(float x) {
    if (std::isnan(x)) return 0;
    return x >= 65535.0f ? 65535 : x <= 0.0f ? 0 : (uint16_t)x;
}
float quantize_i16(const float* src, size_t n, float max, int16_t* dst) {
    if (!(max > 0.0f && std::isfinite(max))) { std::fill(dst, dst + n, (int16_t)0); return 0.0f; }
    const float k = 32767.0f / max;
    for (size_t i = 0; i < n; i++) dst[i] = sat_i16(std::nearbyint(src[i] * k));
    return max;
}
float quantize_u16(const float* src, size_t n, float max, uint16_t* dst) {
    if (!(max > 0.0f && std::isfinite(max))) { std::fill(dst, dst + n, (uint16_t)0); return 0.0f; }
    const float k = 65535.0f / max;
    for (size_t i = 0; i < n; i++) dst[i] = sat_u16(std::nearbyint(std::fmax(src[i], 0.0f) * k));
    return max;
}
float encode_i16(const float* src, size_t n, int16_t* dst) {
    float m = 0.0f;
    for (size_t i = 0; i < n; i++) m = std::fmax(m, std::fabs(src[i]));
    return quantize_i16(src, n, m, dst);
}
float encode_u16(const float* src, size_t n, uint16_t* dst) {
    float m = 0.0f;
    for (size_t i = 0; i < n; i++) m = std::fmax(m, src[i]);
    return quantize_u16(src, n, m, dst);
}
void decode_i16(const int16_t* q, size_t n, float scale, float* out) {
    const float k = scale / 32767.0f;
    for (size_t i = 0; i < n; i++) out[i] = (float)q[i] * k;
}
void decode_u16(const uint16_t* q, size_t n, float scale, float* out) {
    const float k = scale / 65535.0f;
    for (size_t i = 0; i < n; i++) out[i] = (float)q[i] * k;
}

void Arena::init(int k, uint64_t len, size_t nodes) {
    kind = k;
    f.clear(); qi.clear(); qu.clear(); scale.clear();
    if (k == 0) f.assign(len, 0.0f);
    else if (k == 1) { qi.assign(len, 0); scale.assign(nodes, 0.0f); }
    else { qu.assign(len, 0); scale.assign(nodes, 0.0f); }
}
size_t Arena::bytes() const { return f.size() * 4 + qi.size() * 2 + qu.size() * 2 + scale.size() * 4; }
void Arena::read(uint32_t node, uint64_t off, size_t n, float* out) const {
    if (kind == 0) std::memcpy(out, f.data() + off, n * sizeof(float));
    else if (kind == 1) decode_i16(qi.data() + off, n, scale[node], out);
    else decode_u16(qu.data() + off, n, scale[node], out);
}
void Arena::write(uint32_t node, uint64_t off, size_t n, const float* src) {
    if (kind == 0) std::memcpy(f.data() + off, src, n * sizeof(float));
    else if (kind == 1) scale[node] = encode_i16(src, n, qi.data() + off);
    else scale[node] = encode_u16(src, n, qu.data() + off);
}

// --------------------------------------------------------------- HostSolver
HostSolver::HostSolver(std::shared_ptr<Spot> s, int storage_mode, int algorithm, bool iso, bool with_arenas)
    : spot(std::move(s)), storage(storage_mode), algo(algorithm), use_iso(iso) {
    const size_t nn = spot->tree.size();
    if (!with_arenas) return;
    for (int p = 0; p < 2; p++) {
        regrets[p].init(storage == kStoreF32 ? 0 : 1, spot->tree.data_size[p], nn);
        strat[p].init(storage == kStoreF32 ? 0 : 2, spot->tree.data_size[p], nn);
    }
}
void HostSolver::ensure_preds() {  // cfr.rs:157-168
    if (have_preds) return;
    for (int p = 0; p < 2; p++) preds[p].init(storage == kStoreF32 ? 0 : 1, spot->tree.data_size[p], spot->tree.size());
    have_preds = true;
}
uint64_t HostSolver::arena_bytes() const {
    uint64_t b = 0;
    for (int p = 0; p < 2; p++) b += regrets[p].bytes() + strat[p].bytes() + (have_preds ? preds[p].bytes() : 0);
    return b;
}
static Arena& pick(HostSolver& s, int which, int p) {
    if (which == kPreds) { s.ensure_preds(); return s.preds[p]; }
    return which == kRegrets ? s.regrets[p] : s.strat[p];
}
void HostSolver::arena_f32(int which, int p, float* out) const {  // save.rs:76-90
    const Tree& t = spot->tree;
    const size_t nh = spot->hands[p].size();
    std::memset(out, 0, sizeof(float) * t.data_size[p]);
    if (which == kPreds && !have_preds) return;
    const Arena& a = which == kRegrets ? regrets[p] : which == kStrategy ? strat[p] : preds[p];
    for (uint32_t n = 0; n < t.size(); n++)
        if (t.kind[n] == kAction && t.player[n] == p) a.read(n, t.data_off[n], t.nchild[n] * nh, out + t.data_off[n]);
}
void HostSolver::set_arena_f32(int which, int p, const float* in) {
    arenas_zero = false;
    const Tree& t = spot->tree;
    const size_t nh = spot->hands[p].size();
    Arena& a = pick(*this, which, p);
    for (uint32_t n = 0; n < t.size(); n++)
        if (t.kind[n] == kAction && t.player[n] == p) a.write(n, t.data_off[n], t.nchild[n] * nh, in + t.data_off[n]);
}
void HostSolver::solved_strategy(uint32_t node, float* sig) const {  // cfr.rs:679-726
    const Tree& t = spot->tree;
    const int p = t.player[node], na = t.nchild[node];
    const int nh = (int)spot->hands[p].size();
    const Arena& a = strat[p];
    const uint64_t off = t.data_off[node];
    for (int i = 0; i < nh; i++) {
        if (a.kind == 0) {
            double sum = 0;
            for (int k = 0; k < na; k++) sum += (double)std::fmax(a.f[off + k * nh + i], 0.0f);
            for (int k = 0; k < na; k++)
                sig[k * nh + i] = sum > 1e-12 ? (float)((double)std::fmax(a.f[off + k * nh + i], 0.0f) / sum)
                                              : 1.0f / (float)na;
        } else {
            uint32_t sum = 0;
            for (int k = 0; k < na; k++) sum += a.qu[off + k * nh + i];
            const float inv = sum > 0 ? 1.0f / (float)sum : 0.0f;
            for (int k = 0; k < na; k++)
                sig[k * nh + i] = sum > 0 ? (float)a.qu[off + k * nh + i] * inv : 1.0f / (float)na;
        }
    }
}
void HostSolver::average_strategy(uint32_t node, float* sig) const {
    auto it = locks.find(node);
    if (it != locks.end()) { std::memcpy(sig, it->second.data(), it->second.size() * sizeof(float)); return; }
    solved_strategy(node, sig);
}

// -------------------------------------------------- symmetrise (cfr.rs:749-871)
void HostSolver::ensure_symmetric() {
    if (!sym_dirty || !use_iso || spot->perms.size() < 2) { sym_dirty = false; return; }
    arenas_zero = false;
    sym_walk(0, nullptr, 0, [&](uint32_t src, uint32_t dst, int k) { copy_branch(src, dst, k); });
    sym_dirty = false;
}
// The branch copies of ensure_symmetric in its order (cfr.rs:749-800): below
// every chance node, the representative children first (recursively), then
// each non-representative child from its representative with the first
// permutation that maps the card onto it.
void HostSolver::sym_walk(uint32_t node, const uint8_t* dealt, int nd,
                          const std::function<void(uint32_t, uint32_t, int)>& on_branch) const {
    const Tree& t = spot->tree;
    if (t.kind[node] == kAction) {
        for (int a = 0; a < t.nchild[node]; a++) sym_walk(t.child(node, a), dealt, nd, on_branch);
        return;
    }
    if (t.kind[node] != kChance) return;
    std::vector<int> valid = spot->perms_fixing(dealt, nd);
    struct O { uint8_t c, rep; int k; };
    std::vector<O> orbit;
    for (int c = 0; c < 52; c++) {
        bool was = false;
        for (int i = 0; i < nd; i++) was = was || dealt[i] == c;
        if (t.children[t.child_start[node] + c] == kSentinel || was) continue;
        uint8_t rep = (uint8_t)c;
        int kr = 0;
        for (int k : valid) {
            uint8_t pc = card_permute((uint8_t)c, spot->perms[k]);
            if (pc < rep) { rep = pc; kr = k; }
        }
        orbit.push_back({(uint8_t)c, rep, kr});
    }
    uint8_t d2[2] = {nd > 0 ? dealt[0] : (uint8_t)0, 0};
    for (auto& o : orbit)
        if (o.c == o.rep) {
            d2[nd] = o.c;
            sym_walk(t.children[t.child_start[node] + o.c], d2, nd + 1, on_branch);
        }
    for (auto& o : orbit)
        if (o.c != o.rep) on_branch(t.children[t.child_start[node] + o.rep], t.children[t.child_start[node] + o.c], o.k);
}
// The action-node pairs of one branch copy, parent before children
// (cfr.rs:806-871).
void HostSolver::branch_walk(uint32_t src, uint32_t dst, int k, const std::function<void(uint32_t, uint32_t)>& on_action) const {
    const Tree& t = spot->tree;
    if (t.kind[src] == kAction) {
        on_action(src, dst);
        for (int a = 0; a < t.nchild[src]; a++) branch_walk(t.child(src, a), t.child(dst, a), k, on_action);
    } else if (t.kind[src] == kChance) {
        for (int x = 0; x < 52; x++) {
            uint32_t dc = t.children[t.child_start[dst] + x];
            if (dc == kSentinel) continue;
            uint8_t sx = card_permute((uint8_t)x, spot->perms[k]);
            branch_walk(t.children[t.child_start[src] + sx], dc, k, on_action);
        }
    }
}
void HostSolver::copy_branch(uint32_t src, uint32_t dst, int k) {
    const Tree& t = spot->tree;
    branch_walk(src, dst, k, [&](uint32_t s, uint32_t d) {
        const int p = t.player[s], na = t.nchild[s];
        const size_t nh = spot->hands[p].size(), cnt = na * nh;
        const auto& tbl = spot->hand_perm[p][k];
        auto lk = locks.find(s);
        std::vector<float> sr(cnt), ss(cnt), dr(cnt), ds(cnt);
        regrets[p].read(s, t.data_off[s], cnt, sr.data());
        strat[p].read(s, t.data_off[s], cnt, ss.data());
        for (int a = 0; a < na; a++)
            for (size_t i = 0; i < nh; i++) {
                size_t j = tbl[i];
                dr[a * nh + i] = sr[a * nh + j];
                ds[a * nh + i] = lk != locks.end() ? lk->second[a * nh + j] : ss[a * nh + j];
            }
        regrets[p].write(d, t.data_off[d], cnt, dr.data());
        strat[p].write(d, t.data_off[d], cnt, ds.data());
    });
}
std::vector<HostSolver::SymCopy> HostSolver::symmetric_copies() const {
    std::vector<SymCopy> out;
    if (!use_iso || spot->perms.size() < 2) return out;
    sym_walk(0, nullptr, 0, [&](uint32_t src, uint32_t dst, int k) {
        branch_walk(src, dst, k, [&](uint32_t s, uint32_t d) { out.push_back({s, d, k}); });
    });
    return out;
}

// ------------------------------------------------------- locks (query.rs)
std::vector<float> normalize_freqs(const std::vector<float>& f, int na) {  // query.rs:40-61
    if ((int)f.size() != na)
        throw Error("expected " + std::to_string(na) + " action frequencies, got " + std::to_string(f.size()));
    double sum = 0;
    for (float x : f) {
        if (x < 0.0f || !std::isfinite(x)) throw Error("frequencies must be finite and >= 0");
        sum += (double)x;
    }
    if (!std::isfinite(sum) || sum > 1e9)
        throw Error("frequencies sum to more than 1e9 -- not a frequency vector (use values on a 0..1 scale)");
    if (sum <= 1e-9) throw Error("at least one frequency must be positive");
    std::vector<float> out(f.size());
    for (size_t i = 0; i < f.size(); i++) out[i] = (float)((double)f[i] / sum);
    return out;
}
void rake_to_target(float* sg, int na, int nh, const float* reach, const float* target) {  // query.rs:68-156
    std::vector<double> m(na);
    for (int a = 0; a < na; a++) m[a] = target[a] > 1e-9f ? 1.0 : 0.0;
    for (int i = 0; i < nh; i++) {
        double mass = 0;
        for (int a = 0; a < na; a++)
            if (target[a] > 1e-9f) mass += (double)sg[a * nh + i];
        if (mass <= 1e-12)
            for (int a = 0; a < na; a++) sg[a * nh + i] = target[a];
    }
    std::vector<double> agg(na);
    for (int round = 0; round < 400; round++) {
        std::fill(agg.begin(), agg.end(), 0.0);
        double total = 0;
        for (int i = 0; i < nh; i++) {
            const double w = reach[i];
            if (w <= 0.0) continue;
            double den = 0;
            for (int a = 0; a < na; a++) den += m[a] * (double)sg[a * nh + i];
            if (den <= 1e-12) continue;
            total += w;
            for (int a = 0; a < na; a++) agg[a] += w * m[a] * (double)sg[a * nh + i] / den;
        }
        if (total <= 1e-12) break;
        double err = 0;
        for (int a = 0; a < na; a++) {
            if (target[a] <= 1e-9f) continue;
            const double f = agg[a] / total;
            err = std::max(err, std::fabs(f - (double)target[a]));
            if (f > 1e-9) m[a] *= (double)target[a] / f;
        }
        double ms = 0;
        for (double x : m) ms += x;
        if (ms > 1e-12)
            for (auto& x : m) x *= (double)na / ms;
        if (err < 1e-4) break;
    }
    for (int i = 0; i < nh; i++) {
        double s = 0;
        for (int a = 0; a < na; a++) {
            const double v = m[a] * (double)sg[a * nh + i];
            sg[a * nh + i] = (float)v;
            s += v;
        }
        for (int a = 0; a < na; a++) sg[a * nh + i] = s > 1e-12 ? (float)((double)sg[a * nh + i] / s) : target[a];
    }
}
std::vector<int> HostSolver::canonical_steps(const std::vector<int>& steps, std::array<uint8_t, 4>* perm) const {
    // query.rs:667-697
    std::array<uint8_t, 4> comp = {0, 1, 2, 3};
    std::vector<int> out = steps;
    if (use_iso && spot->perms.size() >= 2) {
        uint8_t dealt[2];
        int nd = 0;
        for (auto& s : out) {
            if (s >= 0) continue;
            const uint8_t cm = card_permute((uint8_t)(-1 - s), comp);
            uint8_t rep = cm;
            int kr = -1;
            for (int k : spot->perms_fixing(dealt, nd)) {
                uint8_t pc = card_permute(cm, spot->perms[k]);
                if (pc < rep) { rep = pc; kr = k; }
            }
            if (kr >= 0)
                for (auto& x : comp) x = spot->perms[kr][x];
            if (nd < 2) dealt[nd++] = rep;
            s = -1 - (int)rep;
        }
    }
    if (perm) *perm = comp;
    return out;
}
void HostSolver::walk(const std::vector<int>& steps, uint32_t* node_out, std::vector<float> reach[2]) const {
    // query.rs:304-340
    const Tree& t = spot->tree;
    uint32_t n = 0;
    reach[0] = spot->hands[0].w;
    reach[1] = spot->hands[1].w;
    uint8_t dealt[2];
    int nd = 0;
    for (int s : steps) {
        if (t.kind[n] == kAction && s >= 0) {
            const int na = t.nchild[n], p = t.player[n];
            if (s >= na) throw Error("action index " + std::to_string(s) + " out of range");
            const size_t nh = spot->hands[p].size();
            std::vector<float> sig(na * nh);
            average_strategy(n, sig.data());
            for (size_t i = 0; i < nh; i++) reach[p][i] *= sig[s * nh + i];
            n = t.child(n, s);
        } else if (t.kind[n] == kChance && s < 0) {
            const uint8_t c = (uint8_t)(-1 - s);
            bool was = false;
            for (int i = 0; i < nd; i++) was = was || dealt[i] == c;
            const uint32_t ch = t.children[t.child_start[n] + c];
            if (ch == kSentinel || was) throw Error("card " + card_name(c) + " not available here");
            for (int p = 0; p < 2; p++)
                for (size_t i = 0; i < spot->hands[p].size(); i++)
                    if (spot->hands[p].mask[i] >> c & 1) reach[p][i] = 0.0f;
            if (nd < 2) dealt[nd++] = c;
            n = ch;
        } else {
            throw Error("path step does not match the node kind");
        }
    }
    *node_out = n;
}
uint32_t HostSolver::lock_node(const std::vector<int>& steps, int mode, const std::vector<float>& freqs,
                               const std::vector<std::pair<std::string, std::vector<float>>>& edits,
                               const std::string& label) {  // query.rs:700-773
    std::array<uint8_t, 4> perm;
    std::vector<int> canon = canonical_steps(steps, &perm);
    uint32_t node;
    std::vector<float> reach[2];
    walk(canon, &node, reach);
    const Tree& t = spot->tree;
    if (t.kind[node] != kAction) throw Error("only action nodes can be locked");
    const int na = t.nchild[node], p = t.player[node];
    const int nh = (int)spot->hands[p].size();
    std::vector<float> sig((size_t)na * nh);
    if (mode == 0) {
        solved_strategy(node, sig.data());
    } else if (mode == 1) {
        std::vector<float> tgt = normalize_freqs(freqs, na);
        solved_strategy(node, sig.data());
        rake_to_target(sig.data(), na, nh, reach[p].data(), tgt.data());
    } else {
        average_strategy(node, sig.data());
        for (auto& e : edits) {
            std::vector<float> tgt = normalize_freqs(e.second, na);
            std::vector<uint8_t> cc = parse_board(e.first);
            if (cc.size() != 2) throw Error("expected a 2-card combo, got \"" + e.first + "\"");
            const uint8_t c1 = card_permute(cc[0], perm), c2 = card_permute(cc[1], perm);
            int idx = -1;
            for (int i = 0; i < nh && idx < 0; i++) {
                const uint8_t h1 = spot->hands[p].c1[i], h2 = spot->hands[p].c2[i];
                if ((h1 == c1 && h2 == c2) || (h1 == c2 && h2 == c1)) idx = i;
            }
            if (idx < 0) throw Error(e.first + " is not in " + (p == 0 ? "OOP" : "IP") + "'s range here");
            for (int a = 0; a < na; a++) sig[(size_t)a * nh + idx] = tgt[a];
        }
    }
    locks[node] = std::move(sig);
    lock_labels[node] = label;
    sym_dirty = true;
    return node;
}
void validate_locks(const Spot& spot, const std::vector<std::pair<uint32_t, std::vector<float>>>& locks) {
    // save.rs:45-72
    const Tree& t = spot.tree;
    for (auto& l : locks) {
        const uint32_t idx = l.first;
        if (idx >= t.size())
            throw Error("lock at node " + std::to_string(idx) + ": index out of range (tree has " +
                        std::to_string(t.size()) + " nodes)");
        if (t.kind[idx] != kAction) throw Error("lock at node " + std::to_string(idx) + ": not an action node");
        const size_t want = (size_t)t.nchild[idx] * spot.hands[t.player[idx]].size();
        if (l.second.size() != want)
            throw Error("lock at node " + std::to_string(idx) + ": sigma has " + std::to_string(l.second.size()) +
                        " entries, expected " + std::to_string(want));
        for (float v : l.second)
            if (!std::isfinite(v) || v < 0.0f)
                throw Error("lock at node " + std::to_string(idx) + ": invalid frequency (must be finite and >= 0)");
    }
}

// ------------------------------------------------------------ .gto (save.rs)
static const char kMagic[] = "GTOSOLVE2\n";

void HostSolver::save(const std::string& path) const {  // save.rs:92-143
    std::vector<float> buf;
    save_stream(path, iteration, [&](int k, FILE* f) {
        const int p = k % 2, which = k < 2 ? kRegrets : kStrategy;
        const uint64_t len = spot->tree.data_size[p];
        buf.resize(len);
        arena_f32(which, p, buf.data());
        return write_arena_len(f, len) && fwrite(buf.data(), 4, len, f) == len;
    });
}
bool write_arena_len(FILE* f, uint64_t len) {
    uint8_t lenb[8];
    for (int b = 0; b < 8; b++) lenb[b] = (uint8_t)(len >> (8 * b));
    return fwrite(lenb, 1, 8, f) == 8;
}
void HostSolver::save_stream(const std::string& path, uint32_t iter,
                             const std::function<bool(int, FILE*)>& write_arena) const {
    const std::string tmp = path + ".tmp";
    auto fail = [&](const std::string& m) {
        std::remove(tmp.c_str());
        throw Error(m);
    };
    FILE* f = fopen(tmp.c_str(), "wb");
    if (!f) throw Error("cannot create " + tmp + ": " + strerror(errno));
    json::Value h = json::Value::object();
    h.set("config", config_to_json(spot->config));
    h.set("iteration", json::Value::integer(iter));
    json::Value lk = json::Value::array(), lb = json::Value::array();
    for (auto& kv : locks) {
        json::Value e = json::Value::array(), s = json::Value::array();
        e.arr.push_back(json::Value::integer(kv.first));
        for (float x : kv.second) s.arr.push_back(json::Value::f32(x));
        e.arr.push_back(s);
        lk.arr.push_back(e);
    }
    for (auto& kv : lock_labels) {
        json::Value e = json::Value::array();
        e.arr.push_back(json::Value::integer(kv.first));
        e.arr.push_back(json::Value::string(kv.second));
        lb.arr.push_back(e);
    }
    h.set("locks", lk);
    h.set("lock_labels", lb);
    std::string hs = json::dump(h);
    bool ok = fwrite(kMagic, 1, 10, f) == 10 && fwrite(hs.data(), 1, hs.size(), f) == hs.size() && fputc('\n', f) != EOF;
    try {
        for (int k = 0; k < 4 && ok; k++) ok = write_arena(k, f);
    } catch (...) {
        fclose(f);
        std::remove(tmp.c_str());
        throw;
    }
    ok = ok && fflush(f) == 0 && fsync(fileno(f)) == 0;
    if (fclose(f) != 0) ok = false;
    if (!ok) fail("write failed: " + tmp);
    if (std::rename(tmp.c_str(), path.c_str()) != 0) fail("rename failed: " + std::string(strerror(errno)));
}

std::unique_ptr<HostSolver> HostSolver::load(const std::string& path, int storage_mode) {  // save.rs:149-227
    std::ifstream in(path, std::ios::binary);
    if (!in) throw Error("cannot open " + path);
    auto s = load_header(in, storage_mode);
    const Spot* spot = s->spot.get();
    s->arenas_zero = false;
    std::vector<float> buf;
    for (int k = 0; k < 4; k++) {
        const int p = k % 2;
        const uint64_t len = read_arena_len(in, spot->tree.data_size[p]);
        buf.resize(len);
        if (!in.read((char*)buf.data(), (std::streamsize)(len * 4))) throw Error("truncated arena");
        s->set_arena_f32(k < 2 ? kRegrets : kStrategy, p, buf.data());
    }
    return s;
}
uint64_t read_arena_len(std::istream& in, uint64_t expected) {
    uint8_t lb[8];
    if (!in.read((char*)lb, 8)) throw Error("truncated arena");
    uint64_t len = 0;
    for (int b = 0; b < 8; b++) len |= (uint64_t)lb[b] << (8 * b);
    if (len != expected)
        throw Error("arena size mismatch: file " + std::to_string(len) + ", expected " + std::to_string(expected) +
                    " (tree config changed?)");
    return len;
}
std::unique_ptr<HostSolver> HostSolver::load_header(std::istream& in, int storage_mode) {  // save.rs:149-188
    char magic[10];
    if (!in.read(magic, 10) || std::memcmp(magic, kMagic, 10) != 0) throw Error("not a solver save file");
    std::string hl;
    if (!std::getline(in, hl)) throw Error("truncated header");
    json::Value h;
    try {
        h = json::parse(hl);
    } catch (const std::exception& e) {
        throw Error(std::string("bad header: ") + e.what());
    }
    const json::Value* cfg = h.get("config");
    const json::Value* it = h.get("iteration");
    if (!cfg || !it || it->kind != json::Value::NUM) throw Error("bad header: missing config or iteration");
    std::shared_ptr<Spot> spot(build_spot(config_from_json(*cfg), 0, /*lenient=*/true).release());
    std::vector<std::pair<uint32_t, std::vector<float>>> locks;
    std::map<uint32_t, std::string> labels;
    if (const json::Value* l = h.get("locks")) {
        for (auto& e : l->arr) {
            if (e.kind != json::Value::ARR || e.arr.size() != 2 || e.arr[0].kind != json::Value::NUM ||
                e.arr[1].kind != json::Value::ARR)
                throw Error("bad header: malformed lock entry");
            std::vector<float> s;
            for (auto& x : e.arr[1].arr) {
                if (x.kind != json::Value::NUM) throw Error("bad lock section: non-numeric frequency");
                s.push_back((float)x.num);
            }
            locks.push_back({(uint32_t)e.arr[0].num, s});
        }
    }
    if (const json::Value* l = h.get("lock_labels"))
        for (auto& e : l->arr)
            if (e.kind == json::Value::ARR && e.arr.size() == 2 && e.arr[1].kind == json::Value::STR)
                labels[(uint32_t)e.arr[0].num] = e.arr[1].str;
    try {
        validate_locks(*spot, locks);
    } catch (const Error& e) {
        throw Error(std::string("bad lock section: ") + e.what());
    }
    auto s = std::make_unique<HostSolver>(spot, storage_mode, kDcfr, true);
    s->iteration = (uint32_t)it->num;
    for (auto& l : locks) s->locks[l.first] = l.second;
    s->lock_labels = labels;
    if (!s->locks.empty()) s->sym_dirty = true;
    return s;
}

}  // namespace gtob
