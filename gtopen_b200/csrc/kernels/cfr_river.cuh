// River programs: one CTA solves a whole river betting round (every action
// node, fold and showdown below a river deal) depth first, the way the
// reference's CPU recursion walks it (cfr.rs:414-534), with the vectors of
// the current path in shared memory.  Reach vectors below the round's root
// and the children's values never touch HBM: a sweep reads each visited
// arena block once (the traverser's regret and strategy-sum blocks are read
// and written once) plus the two reach vectors at the root and writes the
// root's value, instead of a level-synchronous sweep's per-node reach and cfv
// slots.
//
// The walk is the plan's step list (plan.hpp RStep).  Per depth d of the
// current path the CTA keeps: the reach vector that changed entering d (the
// opponent's below an opponent node, the traverser's below one of its own),
// the node's staged sigma-source block(s), and -- at the traverser's depths --
// one value row per child (the update needs every child's value).  An
// opponent node's children add their values, in child order, straight into
// its row of the traverser parent's value rows (or into a root buffer).
//
// Arena blocks arrive by bulk asynchronous copies (cp.async.bulk, no
// multicast) into a ring of shared-memory slots, issued by thread 0 up to
// `nslot` blocks ahead of the step that consumes them -- across the CTA's
// next subtree too -- so the walk rarely waits for HBM.  Every wait is bounded
// as in the other staged kernels: a copy that does not land within kWaitNs
// sets bit 0 of Dev::err, the CTA waits (bounded) for its copies in flight
// and ends.
//
// The arithmetic is the staged kernels' (the same device functions: sigma,
// the update, exact fold and showdown sums), so the arenas and values are
// bit-identical to the level-synchronous staged engine's.
#pragma once
#include "cfr_staged.cuh"

namespace gtob {

constexpr int kRiverNT = 256;  // threads of a river CTA

// Shared-memory layout of kr_river (byte offsets), the same on host and device.
struct RLayout {
    int nslot;           // ring slots
    int depth;           // depths held (deepest river action node + 1)
    unsigned slot;       // bytes per ring slot: one block of kSKA x nh_pad entries
    unsigned bars;       // nslot + 1 mbarriers (the last: the showdown tables)
    unsigned ring;
    unsigned root_ro, root_rp, root_acc, tmp;  // f32 vectors of nh_pad
    unsigned vec[kRiverMaxDepth];              // depth >= 1: the reach vector that changed there
    unsigned blk[kRiverMaxDepth];              // the node's sigma-source block, then its predictions
    unsigned val[kRiverMaxDepth];              // the traverser's depths: kSKA value rows
    unsigned tab;                              // showdown tables: entries of the subtree's board
    unsigned u;                                // showdown scan output (long long)
    unsigned total;
};
__host__ __device__ inline unsigned rl_r16(unsigned b) { return (b + 15u) & ~15u; }
// p: the traverser of the sweep (depth d is the traverser's iff (d & 1) == p,
// as the plan checked); msort: the plan's longest strength list.
inline RLayout river_layout(int nh_pad, int esz, bool pcfr, int depth, int p, int msort, int nslot) {
    RLayout L{};
    L.nslot = nslot;
    L.depth = depth;
    L.slot = rl_r16((unsigned)(kSKA * nh_pad * esz));
    const unsigned vec = (unsigned)nh_pad * 4u;
    unsigned o = 0;
    L.bars = o;
    o += rl_r16(8u * (unsigned)(nslot + 1));
    L.ring = o;
    o += (unsigned)nslot * L.slot;
    L.root_ro = o;
    o += vec;
    L.root_rp = o;
    o += vec;
    L.root_acc = o;
    o += vec;
    L.tmp = o;
    o += vec;
    for (int d = 0; d < depth; d++) {
        L.vec[d] = d ? o : 0u;
        if (d) o += vec;
        L.blk[d] = o;
        o += L.slot * (pcfr ? 2u : 1u);
        L.val[d] = (d & 1) == p ? o : 0u;
        if ((d & 1) == p) o += (unsigned)kSKA * vec;
    }
    L.tab = o;
    o += rl_r16(4u * (56u + 3u * (unsigned)nh_pad));
    L.u = o;
    o += rl_r16(8u * (3u * (unsigned)msort + 53u));
    L.total = o;
    return L;
}

// Per depth of the current path (shared memory, written by thread 0 when the
// node is entered).
struct RDepth {
    uint64_t aoff;
    long long loff;  // lock table offset, -1 = unlocked
    float kr, kp, sscale;
    uint32_t sidx;
    int na, actor, k;
    unsigned ro, rp, acc;  // shared-memory offsets of the reach vectors and of the opponent node's accumulator
};

// Showdown table image of one river board for the hands of player o: 53
// card-list offsets (padded to 56 words), then one word per scan entry as
// load_show_tab builds them (opponent hand | segment start << 12 | output
// index << 16), padded to a multiple of 4 words so every image starts on a
// 16-byte boundary.  Built on the host; one bulk copy per subtree.
__host__ __device__ inline unsigned river_tab_words(int m, int ne) { return 56u + (((unsigned)(m + ne) + 3u) & ~3u); }

// Fold summary (game.rs:478-485) of the opponent reach vector `ro` in shared
// memory whose grid scale sc is known: per-card exact sums S[52] (zeroed by
// the caller before its last barrier) and the total.  NT threads; s_red: NT/32
// long longs.
template <int NT>
__device__ long long r_fold_total(const Dev& d, int o, const float* ro, int sc, long long* S, long long* s_red) {
    constexpr int W = NT / 32;
    const int nho = d.nh[o];
    const uint32_t* hi = d.hinfo[o];
    long long t = 0;
    for (int j = threadIdx.x; j < nho; j += NT) {
        const long long q = fix_q(ro[j], sc);
        if (q) {
            const uint32_t h = hi[j];
            t += q;
            atomicAdd((unsigned long long*)&S[h & 63u], (unsigned long long)q);
            atomicAdd((unsigned long long*)&S[(h >> 6) & 63u], (unsigned long long)q);
        }
    }
#pragma unroll
    for (int x = 16; x > 0; x >>= 1) t += __shfl_xor_sync(0xffffffffu, t, x);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = t;
    __syncthreads();
    long long total = 0;
#pragma unroll
    for (int k = 0; k < W; k++) total += s_red[k];
    return total;
}

// One showdown (game.rs:501-577) of the opponent reach `ro` (grid scale sc)
// against the board's tables tb: the segmented scan of cta_showdown2 on one
// vector, then the traverser's rank entries.  Values go to out[hand] (added
// when acc_out; hands blocked by the board get 0).  Ends without a barrier.
template <int NT>
__device__ void r_showdown(const ShowTab& tb, int msort, const float* ro, int sc, float twin, float tlose, float ttie,
                           float* out, bool acc_out, long long* U, long long* s_w, int* s_wf) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m = tb.m;
    const int F = m + tb.ne;
    const int chunk = ((F + NT - 1) / NT) | 1;
    const int f0 = min(tid * chunk, F), f1 = min(f0 + chunk, F);
    long long ax = 0;
    bool seen = false;
    for (int f = f0; f < f1; f++) {
        const uint32_t en = tb.ent[f];
        if ((en >> 12) & 1u) {
            ax = 0;
            seen = true;
        }
        ax += fix_q(ro[en & 0xFFFu], sc);
        U[en >> 16] = ax;
    }
    if (tid == 0) U[0] = 0;
    if (tid < 52) U[msort + 1 + tb.coff[tid] + tid] = 0;
    bool fl = seen;
    long long sx = ax;
#pragma unroll
    for (int x = 1; x < 32; x <<= 1) {
        const int fu = __shfl_up_sync(0xffffffffu, (int)fl, x);
        const long long ux = __shfl_up_sync(0xffffffffu, sx, x);
        if (lane >= x) {
            if (!fl) sx += ux;
            fl = fl || fu;
        }
    }
    int ef = __shfl_up_sync(0xffffffffu, (int)fl, 1);
    long long ex = __shfl_up_sync(0xffffffffu, sx, 1);
    if (lane == 0) {
        ef = 0;
        ex = 0;
    }
    if (lane == 31) {
        s_w[warp] = sx;
        s_wf[warp] = (int)fl;
    }
    __syncthreads();
    long long cx = 0;
    for (int k = 0; k < warp; k++) cx = s_wf[k] ? s_w[k] : cx + s_w[k];
    cx = ef ? ex : cx + ex;
    if (cx) {
        for (int f = f0; f < f1; f++) {
            const uint32_t en = tb.ent[f];
            if ((en >> 12) & 1u) break;
            U[en >> 16] += cx;
        }
    }
    __syncthreads();
    const long long total = U[m];
    const long long* Q = U + msort + 1;
    for (int k = tid; k < tb.mp; k += NT) {
        const RankEntry e = tb.rank[k];
        const int a1 = e.cards & 0xFF, a2 = e.cards >> 8;
        const long long plb = U[e.lb], pub = U[e.ub], q1lo = Q[e.q1lo], q2lo = Q[e.q2lo], q1hi = Q[e.q1hi],
                        q2hi = Q[e.q2hi], s1 = Q[tb.coff[a1 + 1] + a1], s2 = Q[tb.coff[a2 + 1] + a2];
        const uint32_t sm = tb.same[e.idx];
        const float lower = fix_f(plb - q1lo - q2lo, sc);
        const float higher = fix_f((total - pub) - (s1 - q1hi) - (s2 - q2hi), sc);
        const float same_r = sm != kSentinel ? ro[sm] : 0.0f;
        const float valid = fix_f(total - s1 - s2, sc) + same_r;
        const float tied = valid - lower - higher;
        s_put(out, e.idx, twin * lower + tlose * higher + ttie * tied, acc_out);
    }
    for (int z = tid; z < tb.nz; z += NT) s_put(out, tb.zero[z], 0.0f, acc_out);
}

// Ring blocks a step consumes (the producer and the consumers agree on it):
// an action node's sigma source when it is entered (regrets, plus
// predictions for PCFR+; in evaluation sweeps the strategy sums -- the
// opponent plays its average, and so does the traverser in mode 1), and the
// traverser's strategy sums when its node is left (the update).
template <int EVAL>
__device__ __forceinline__ int r_nfetch(const RStep& st, int p, int mode, bool pcfr) {
    const int a = st.x >> 7;
    if (st.op == kREnter) {
        if (!EVAL) return pcfr ? 2 : 1;
        return (mode == 1 || a != p) ? 1 : 0;
    }
    return (!EVAL && st.op == kRExit && a == p) ? 1 : 0;
}
template <int EVAL>
__device__ __forceinline__ const unsigned char* r_fetch_src(const Arenas& ar, const RStep& st, int b, int esz) {
    const int a = st.x >> 7;
    const void* base = st.op == kRExit ? ar.str[a] : EVAL ? ar.str[a] : b == 0 ? ar.reg[a] : ar.pred[a];
    return (const unsigned char*)base + st.aoff * (uint64_t)esz;
}

// One CTA per resident slot of the device, each taking the subtrees
// blockIdx.x, blockIdx.x + gridDim.x, ... (the plan lists them largest
// first).  EVAL = 0: the CFR sweep of traverser p; 1: an evaluation sweep
// (mode 0 best response, 1 average strategy).
template <int FMT, int EVAL, int NT>
__global__ void __launch_bounds__(NT, 1)
    kr_river(Dev d, Arenas ar, const RTree* trees, const RStep* steps, int ntrees, int p, int mode, int msort,
             RLayout L) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ RDepth s_dep[kRiverMaxDepth];
    __shared__ long long s_S[52];
    __shared__ long long s_redl[NT / 32];
    __shared__ float s_redf[3 * (NT / 32)];
    __shared__ int s_wf[NT / 32];
    const int tid = threadIdx.x;
    const int o = 1 - p;
    const int nhp = d.nh[p], nho = d.nh[o];
    const int esz = fmt_bytes(FMT);
    const bool pcfr = ar.pred[0] != nullptr;
    const int vstride = d.nh_pad;
    const int smode = EVAL ? 1 : 0;  // how the opponent's (and, in CFR sweeps, the traverser's) sigma is formed
    uint64_t* bars = (uint64_t*)(sm + L.bars);
    uint64_t* tbar = bars + L.nslot;
    const unsigned nslot = (unsigned)L.nslot;
    auto F = [&](unsigned off) { return (float*)(sm + off); };
    // producer state (thread 0): the next step to scan for blocks, and the
    // blocks issued; consumer state (every thread): the blocks consumed
    int pf_t = blockIdx.x;
    uint32_t pf_s = 0;
    int pf_b = 0;
    unsigned issued = 0, consumed = 0, tab_uses = 0;
    if (tid == 0) {
        for (unsigned k = 0; k <= nslot; k++) mbar_init(&bars[k], 1);
    }
    __syncthreads();
    auto top_up = [&]() {  // thread 0, at step boundaries
        while (issued < consumed + nslot && pf_t < ntrees) {
            const RTree T = trees[pf_t];
            if (pf_s >= T.step_count) {
                pf_t += gridDim.x;
                pf_s = 0;
                pf_b = 0;
                continue;
            }
            const RStep st = steps[T.step_start + pf_s];
            if (pf_b >= r_nfetch<EVAL>(st, p, mode, pcfr)) {
                pf_s++;
                pf_b = 0;
                continue;
            }
            const int a = st.x >> 7, na = st.x & 0x7F;
            const unsigned bytes = round16((unsigned)(na * d.nh[a] * esz));
            const unsigned slot = issued % nslot;
            mbar_expect_tx(&bars[slot], bytes);
            bulk_load(sm + L.ring + slot * L.slot, r_fetch_src<EVAL>(ar, st, pf_b, esz), bytes, &bars[slot]);
            issued++;
            pf_b++;
        }
    };
    bool tab_pending = false;  // thread 0: a table copy is in flight
    // After a wait that gave up: thread 0 records it and waits (bounded) for
    // every copy still in flight from ring block f on; the CTA then ends.
    auto drain = [&](unsigned f) {
        if (tid != 0) return;
        atomicOr(d.err, 1u);
        for (unsigned g = f; g < issued; g++) mbar_wait(&bars[g % nslot], (g / nslot) & 1u);
        if (tab_pending) mbar_wait(tbar, tab_uses & 1u);
    };
    // Bounded wait for ring block f by every thread; false: the CTA must end.
    auto wait_block = [&](unsigned f) -> bool {
        const bool ok = mbar_wait(&bars[f % nslot], (f / nslot) & 1u);
        if (!__syncthreads_or(!ok)) return true;
        drain(f);
        return false;
    };
    auto step_end = [&]() {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) top_up();
    };
    if (tid == 0) top_up();
    for (int t = blockIdx.x; t < ntrees; t += gridDim.x) {
        const RTree tr = trees[t];
        const uint32_t slot = tr.slot;
        // the board's showdown tables: one bulk copy, waited for at the
        // first showdown (the previous subtree's showdowns are done)
        if (tid == 0) {
            const uint32_t w0 = d.rtab_off[o][slot], nw = d.rtab_off[o][slot + 1] - w0;
            mbar_expect_tx(tbar, nw * 4u);
            bulk_load(sm + L.tab, d.rtab[o] + w0, nw * 4u, tbar);
            tab_pending = true;
        }
        bool tab_ready = false;
        ShowTab tb;
        tb.coff = (const uint32_t*)(sm + L.tab);
        tb.ent = tb.coff + 56;
        tb.m = (int)d.sorted_cnt[o][slot];
        tb.mp = (int)d.rank_cnt[p][slot];
        tb.rank = d.rank[p] + d.rank_off[p][slot];
        const uint32_t z0 = d.zero_off[p][slot];
        tb.nz = (int)(d.zero_off[p][slot + 1] - z0);
        tb.zero = d.zero_idx[p] + z0;
        tb.same = d.same[p];
        // the reach vectors at the root
        {
            const float* g_ro = d.reach[o] + (size_t)tr.rs[o] * d.rstr[o];
            for (int j = tid; j < nho; j += NT) F(L.root_ro)[j] = g_ro[j];
            if (!EVAL) {
                const float* g_rp = d.reach[p] + (size_t)tr.rs[p] * d.rstr[p];
                for (int i = tid; i < nhp; i += NT) F(L.root_rp)[i] = g_rp[i];
            }
        }
        for (uint32_t si = 0; si < tr.step_count; si++) {
            const RStep st = steps[tr.step_start + si];
            const int dep = st.depth;
            if (st.op == kREnter) {
                const int a = st.x >> 7, na = st.x & 0x7F, k = st.k;
                unsigned ro = L.root_ro, rp = L.root_rp, acc = 0;
                if (dep > 0) {
                    // the reach this node's parent passes down action k
                    const RDepth& pd = s_dep[dep - 1];
                    const int pa = pd.actor;
                    ro = pd.ro;
                    rp = pd.rp;
                    if (pa == o || !EVAL) {
                        const unsigned char* b = sm + L.blk[dep - 1];
                        const float* src = F(pa == o ? pd.ro : pd.rp);
                        float* dst = F(L.vec[dep]);
                        const int n = d.nh[pa];
                        float sig[kSKA];
                        for (int i = tid; i < n; i += NT) {
                            s_node_sigma<FMT>(d, pd.loff, pa, i, smode, b, pcfr ? b + L.slot : nullptr, b, pd.kr,
                                              pd.kp, pd.na, sig);
                            dst[i] = src[i] * sig[k];
                        }
                        if (pa == o) ro = L.vec[dep];
                        else rp = L.vec[dep];
                    }
                    if (pa == p) {  // an opponent node: its value accumulates in its parent's row k
                        acc = L.val[dep - 1] + (unsigned)(k * vstride * 4);
                        for (int i = tid; i < nhp; i += NT) F(acc)[i] = 0.0f;
                    }
                } else if (a == o) {
                    acc = L.root_acc;
                    for (int i = tid; i < nhp; i += NT) F(acc)[i] = 0.0f;
                }
                // this node's sigma source (and predictions) out of the ring
                const int nb = r_nfetch<EVAL>(st, p, mode, pcfr);
                for (int b = 0; b < nb; b++) {
                    if (!wait_block(consumed)) return;
                    const int4* sblk = (const int4*)(sm + L.ring + (consumed % nslot) * L.slot);
                    int4* dblk = (int4*)(sm + L.blk[dep] + (unsigned)b * L.slot);
                    const unsigned n16 = round16((unsigned)(na * d.nh[a] * esz)) / 16u;
                    for (unsigned q = tid; q < n16; q += NT) dblk[q] = sblk[q];
                    consumed++;
                }
                if (tid == 0) {
                    RDepth& nd = s_dep[dep];
                    nd.aoff = st.aoff;
                    nd.sidx = st.sidx;
                    nd.na = na;
                    nd.actor = a;
                    nd.k = k;
                    nd.ro = ro;
                    nd.rp = rp;
                    nd.acc = acc;
                    nd.loff = d.lock_off[a][st.sidx];
                    nd.kr = nd.kp = nd.sscale = 0.0f;
                    if (FMT != kDevF32 && nd.loff < 0) {
                        nd.kr = ar.rscale[a][st.sidx] / QT<FMT>::kR;
                        if (pcfr) nd.kp = ar.pscale[a][st.sidx] / QT<FMT>::kR;
                        nd.sscale = ar.sscale[a][st.sidx];
                    }
                }
            }
            else if (st.op == kRFold || st.op == kRShow) {
                // a terminal child k of the node at depth dep
                const RDepth& pd = s_dep[dep];
                const int k = st.k;
                const float twin = __uint_as_float(st.sidx);
                const float tlose = st.pay[0], ttie = st.pay[1];
                // the opponent's reach at the terminal: its own action k
                // taken (the folding player's reach, as the down sweep
                // writes it), or the node's when the traverser acted
                const float* r = F(pd.ro);
                float mx = 0.0f;
                if (pd.actor == o) {
                    const unsigned char* b = sm + L.blk[dep];
                    float* tmp = F(L.tmp);
                    float sig[kSKA];
                    for (int j = tid; j < nho; j += NT) {
                        s_node_sigma<FMT>(d, pd.loff, o, j, smode, b, pcfr ? b + L.slot : nullptr, b, pd.kr, pd.kp,
                                          pd.na, sig);
                        const float v = r[j] * sig[k];
                        tmp[j] = v;
                        mx = fmaxf(mx, v);
                    }
                    r = tmp;
                } else {
                    for (int j = tid; j < nho; j += NT) mx = fmaxf(mx, r[j]);
                }
                if (tid < 52) s_S[tid] = 0;
                mx = warp_max(mx);
                if ((tid & 31) == 0) s_redf[tid >> 5] = mx;
                if (st.op == kRShow && !tab_ready) {  // the board's tables landed?
                    const bool ok = mbar_wait(tbar, tab_uses & 1u);
                    if (__syncthreads_or(!ok)) {
                        drain(consumed);
                        return;
                    }
                    tab_ready = true;
                    if (tid == 0) tab_pending = false;
                    tb.ne = (int)tb.coff[52];
                }
                __syncthreads();
                mx = s_redf[0];
#pragma unroll
                for (int w = 1; w < NT / 32; w++) mx = fmaxf(mx, s_redf[w]);
                const int sc = fix_scale(mx);
                // where the value goes: the traverser's row k, or added to
                // the opponent node's accumulator (children in order)
                const bool add = pd.actor == o;
                float* out = add ? F(pd.acc) : F(L.val[dep]) + k * vstride;
                if (st.op == kRFold) {
                    const long long total = r_fold_total<NT>(d, o, r, sc, s_S, s_redl);
                    const float famount = (int)st.x == p ? tlose : twin;
                    for (int i = tid; i < nhp; i += NT) {
                        const uint32_t h = d.hinfo[p][i];
                        const uint32_t sm_ = h >> 16;
                        const float same_r = sm_ != 0xFFFFu ? r[sm_] : 0.0f;
                        s_put(out, i, famount * (fix_f(total - s_S[h & 63u] - s_S[(h >> 6) & 63u], sc) + same_r),
                              add);
                    }
                } else {
                    r_showdown<NT>(tb, msort, r, sc, twin, tlose, ttie, out, add, (long long*)(sm + L.u), s_redl,
                                   s_wf);
                }
            }
            else {  // kRExit: the node's value to its parent (or the root's slot)
                const RDepth& nd = s_dep[dep];
                float* gout = d.cfv + (size_t)tr.cslot * d.nh_max;
                if (nd.actor == o) {
                    if (dep == 0)
                        for (int i = tid; i < nhp; i += NT) gout[i] = F(nd.acc)[i];
                } else {
                    float* out = dep == 0 ? gout : F(s_dep[dep - 1].acc);
                    const bool add = dep > 0;
                    unsigned char* b_reg = sm + L.blk[dep];
                    unsigned char* b_pred = pcfr ? b_reg + L.slot : nullptr;
                    unsigned char* b_str = b_reg;  // evaluation sweeps: the strategy sums staged on entry
                    if (!EVAL) {
                        if (!wait_block(consumed)) return;
                        b_str = sm + L.ring + (consumed % nslot) * L.slot;
                    }
                    float* cv = F(L.val[dep]);
                    const float* rp = F(nd.rp);
#define RIVER_MINE(NA_)                                                                                            \
    s_mine_node<FMT, EVAL, NA_, NT>(d, ar, p, mode, nd.loff, nd.kr, nd.kp, nd.sscale, nd.sidx, nd.aoff, pcfr, b_reg, \
                                    b_str, b_pred, cv, vstride, rp, out, add, s_redf)
                    switch (nd.na) {
                        case 1: RIVER_MINE(1); break;
                        case 2: RIVER_MINE(2); break;
                        case 3: RIVER_MINE(3); break;
                        default: RIVER_MINE(4); break;
                    }
#undef RIVER_MINE
                    if (!EVAL) consumed++;
                }
            }
            step_end();
        }
        if (!tab_ready) {  // a subtree without showdowns: its table copy still lands before the next
            const bool ok = mbar_wait(tbar, tab_uses & 1u);
            if (__syncthreads_or(!ok)) {
                drain(consumed);
                return;
            }
            if (tid == 0) tab_pending = false;
        }
        tab_uses++;
    }
}

}  // namespace gtob
