// Staged node kernels (the STAGED engine): one CTA per node stages every
// vector and arena block the node needs in shared memory with bulk
// asynchronous copies -- the TMA unit's non-tensor mode, cp.async.bulk --
// that complete on one mbarrier, then computes from shared memory and writes
// its results with 16-byte stores.  All of a node's HBM reads are in flight
// at once (one round trip instead of one per hand chunk and arena field), and
// a 128-thread CTA with ~32 KB of shared memory leaves room for many nodes
// per SM.
//
// Arithmetic is the same as the generic kernels in cfr_kernels.cuh (the same
// expressions in the same order, -fmad=false), so results are identical.
//
// Every wait is bounded: a copy that does not land within kWaitNs sets bit 0
// of Dev::err, waits once more (bounded) for the copies in flight and ends the
// CTA; a source or size the bulk unit cannot take (not 16-byte aligned) sets
// bit 1 and the CTA issues nothing.  The host reads Dev::err at every
// synchronisation point and reports a timeout error.
#pragma once
#include "cfr_kernels.cuh"

namespace gtob {

constexpr int kSThreads = 128;
constexpr int kSWarps = kSThreads / 32;
constexpr int kSKA = 4;                                // staged kernels take nodes with at most 4 actions
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s

// One action node as the staged kernels read it: everything its copies need
// in one 80-byte record (one load round trip per node).
struct alignas(16) SNode {
    uint64_t aoff;             // arena offset (elements) in the actor's arena
    uint32_t cslot, rslot, oslot, sidx;
    uint32_t cs[kSKA];         // child cfv slots (kNoSlot: the fold child)
    uint32_t rs[kSKA];         // child reach slots of the actor (down sweep; kNoSlot: none)
    uint32_t actor, na, fk;    // fk: the fold child's index, kNoSlot if none
    uint32_t folder;           // the folding player of the fold child
    float twin, tlose;         // fold payoffs
};
static_assert(sizeof(SNode) == 80, "SNode layout");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// try_wait with a suspend-time hint: a waiting thread sleeps in the
// instruction (up to kSuspendNs) instead of spinning and issuing.
constexpr unsigned kSuspendNs = 100000u;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity` of the barrier.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity))
        if (globaltimer_ns() - t0 > kWaitNs) return false;
    return true;
}
// Global -> shared bulk copy completing on bar (no multicast).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ unsigned round16(unsigned b) { return (b + 15u) & ~15u; }

// After thread 0 initialised bar and issued the CTA's copies on it (setting
// *s_flag to 1 instead when it refused one as misaligned), every thread
// waits.  Returns false, after the error handling described at the top, when
// the CTA must end.
__device__ bool wait_staged(const Dev& d, uint64_t* bar, int* s_flag) {
    __syncthreads();
    if (*s_flag) return false;
    const bool ok = mbar_wait(bar, 0);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(d.err, 1u);
        if (!ok) mbar_wait(bar, 0);
        return false;
    }
    return true;
}

// 16-byte copy of a staged block back to global memory.
__device__ __forceinline__ void store_block(void* gdst, const void* sblk, unsigned bytes) {
    int4* g = (int4*)gdst;
    const int4* s = (const int4*)sblk;
    for (unsigned k = threadIdx.x; k < bytes / 16; k += blockDim.x) g[k] = s[k];
}

// Strategies of hand i from staged blocks (same expressions as regret_sigma /
// average_sigma in cfr_kernels.cuh).
template <int FMT>
__device__ __forceinline__ void s_regret_sigma(const void* reg, const void* pred, float kr, float kp, int na, int i,
                                               float (&sig)[kSKA]) {
    const int base = i * na;
    float sum = 0.0f;
    if (FMT == kDevF32) {
        const float* r = (const float*)reg + base;
        const float* pr = (const float*)pred;
#pragma unroll
        for (int k = 0; k < kSKA; k++)
            if (k < na) {
                float v = r[k];
                if (pr) v = fmaxf(v, 0.0f) + pr[base + k];
                sig[k] = v;
                sum += fmaxf(v, 0.0f);
            }
    } else if (FMT == kDevFP8) {
        // FP8: regret matching on the stored values before scaling (one scale
        // per node cancels); PCFR+ predictions decoded with their scales
        const uint8_t* q = (const uint8_t*)reg + base;
        const uint8_t* qp = (const uint8_t*)pred;
#pragma unroll
        for (int k = 0; k < kSKA; k++)
            if (k < na) {
                const float v = qp ? fmaxf(e4m3_to_f32(q[k]), 0.0f) * kr + e4m3_to_f32(qp[base + k]) * kp
                                   : e4m3_to_f32(q[k]);
                sig[k] = v;
                sum += fmaxf(v, 0.0f);
            }
    } else {
        const int16_t* q = (const int16_t*)reg + base;
        if (pred) {
            const int16_t* qp = (const int16_t*)pred + base;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) {
                    sig[k] = (float)max((int)q[k], 0) * kr + (float)qp[k] * kp;
                    sum += fmaxf(sig[k], 0.0f);
                }
        } else {
            int isum = 0;
            int qv[kSKA];
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) {
                    qv[k] = max((int)q[k], 0);
                    isum += qv[k];
                }
            if (isum > 0) {
                const float inv = __frcp_rn((float)isum);  // = 1.0f / x, correctly rounded
#pragma unroll
                for (int k = 0; k < kSKA; k++)
                    if (k < na) sig[k] = (float)qv[k] * inv;
            } else {
                const float u = 1.0f / (float)na;
#pragma unroll
                for (int k = 0; k < kSKA; k++)
                    if (k < na) sig[k] = u;
            }
            return;
        }
    }
    if (sum > 1e-12f) {
        const float inv = __frcp_rn(sum);
#pragma unroll
        for (int k = 0; k < kSKA; k++)
            if (k < na) sig[k] = fmaxf(sig[k], 0.0f) * inv;
    } else {
        const float u = 1.0f / (float)na;
#pragma unroll
        for (int k = 0; k < kSKA; k++)
            if (k < na) sig[k] = u;
    }
}
template <int FMT>
__device__ __forceinline__ void s_average_sigma(const void* str, int na, int i, float (&sig)[kSKA]) {
    const int base = i * na;
    if (FMT == kDevF32 || FMT == kDevFP8) {  // FP8: the f32 rule on the stored values (the scale cancels)
        double sum = 0.0;
        float v[kSKA];
#pragma unroll
        for (int k = 0; k < kSKA; k++)
            if (k < na) {
                v[k] = FMT == kDevF32 ? fmaxf(((const float*)str)[base + k], 0.0f)
                                      : fmaxf(e4m3_to_f32(((const uint8_t*)str)[base + k]), 0.0f);
                sum += (double)v[k];
            }
        if (sum > 1e-12) {
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) sig[k] = (float)((double)v[k] / sum);
        } else {
            const float u = 1.0f / (float)na;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) sig[k] = u;
        }
    } else {
        const uint16_t* q = (const uint16_t*)str + base;
        unsigned sum = 0;
        unsigned qv[kSKA];
#pragma unroll
        for (int k = 0; k < kSKA; k++)
            if (k < na) {
                qv[k] = q[k];
                sum += qv[k];
            }
        if (sum > 0) {
            const float inv = __frcp_rn((float)sum);
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) sig[k] = (float)qv[k] * inv;
        } else {
            const float u = 1.0f / (float)na;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) sig[k] = u;
        }
    }
}
template <int FMT>
__device__ __forceinline__ void s_node_sigma(const Dev& d, long long loff, int a, int i, int mode, const void* reg,
                                             const void* pred, const void* str, float kr, float kp, int na,
                                             float (&sig)[kSKA]) {
    if (loff >= 0) {
        const int nh = d.nh[a];
#pragma unroll
        for (int k = 0; k < kSKA; k++)
            if (k < na) sig[k] = d.lock_sig[loff + (long long)k * nh + i];
    } else if (mode == 0) {
        s_regret_sigma<FMT>(reg, pred, kr, kp, na, i, sig);
    } else {
        s_average_sigma<FMT>(str, na, i, sig);
    }
}

// Block maxima of three values behind one barrier (sh: 3 * NT / 32 floats,
// written once per CTA).
template <int NT = kSThreads>
__device__ __forceinline__ void s_block_max3(float& a, float& b, float& c, float* sh) {
    constexpr int W = NT / 32;
    a = warp_max(a);
    b = warp_max(b);
    c = warp_max(c);
    if ((threadIdx.x & 31) == 0) {
        sh[threadIdx.x >> 5] = a;
        sh[W + (threadIdx.x >> 5)] = b;
        sh[2 * W + (threadIdx.x >> 5)] = c;
    }
    __syncthreads();
    a = sh[0];
    b = sh[W];
    c = sh[2 * W];
#pragma unroll
    for (int k = 1; k < W; k++) {
        a = fmaxf(a, sh[k]);
        b = fmaxf(b, sh[W + k]);
        c = fmaxf(c, sh[2 * W + k]);
    }
}

// Fold summary of a staged opponent reach vector (game.rs:478-485), exact
// sums (cfr_kernels.cuh): the vector's grid scale, the total and the
// per-card sums.  Integer sums do not depend on their order, so every thread
// takes hands j = tid, tid + NT, ... and adds each hand's grid value to its
// two cards' sums with shared-memory atomics.  s_red: NT / 32 entries;
// returns the total, *sc_out the scale.
template <int NT = kSThreads>
__device__ long long s_fold_sums(const Dev& d, int o, const float* ro, long long* S, long long* s_red, int* sc_out) {
    constexpr int W = NT / 32;
    const int nho = d.nh[o];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float mx = 0.0f;
    for (int j = threadIdx.x; j < nho; j += NT) mx = fmaxf(mx, ro[j]);
    mx = warp_max(mx);
    float* fred = (float*)s_red;
    if (lane == 0) fred[warp] = mx;
    if (threadIdx.x < 52) S[threadIdx.x] = 0;
    __syncthreads();
    mx = fred[0];
#pragma unroll
    for (int k = 1; k < W; k++) mx = fmaxf(mx, fred[k]);
    const int sc = fix_scale(mx);
    long long t = 0;
    const uint32_t* hi = d.hinfo[o];
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
    __syncthreads();  // every thread has read fred before it is reused as the totals
    if (lane == 0) s_red[warp] = t;
    __syncthreads();
    long long total = 0;
#pragma unroll
    for (int k = 0; k < W; k++) total += s_red[k];
    *sc_out = sc;
    return total;
}

// Shared-memory layout of the staged action kernels (bytes): the regret,
// strategy-sum and (PCFR+ only) prediction blocks, the opponent and own
// reach vectors, then kSKA child value vectors.
// Three layouts: the down kernel (one sigma-source block -- regrets or, in
// evaluation sweeps, strategy sums -- the predictions for PCFR+, the parent
// reach), the up kernel on the traverser's nodes (regret, strategy-sum and
// prediction blocks, opponent and own reach, child values) and the up kernel
// on the opponent's nodes (the fold child's reach, child values).
enum SKind { kSDown = 0, kSUpMine = 1, kSUpOpp = 2 };
struct SLayout {
    unsigned cap, vec, o_str, o_pred, o_ro, o_rp, o_cv, total;
    __host__ __device__ SLayout(int nh_pad, int esz, bool pred, int kind) {
        cap = ((unsigned)(kSKA * nh_pad * esz) + 15u) & ~15u;
        vec = (unsigned)nh_pad * 4u;
        unsigned o = 16;
        if (kind != kSUpOpp) o += cap;  // the first block (regrets / sigma source) starts at 16
        o_str = kind == kSUpMine ? o : 16u;
        if (kind == kSUpMine) o += cap;
        o_pred = o;
        if (pred && kind != kSUpOpp) o += cap;
        o_ro = o;
        o += vec;
        o_rp = o;
        if (kind == kSUpMine) o += vec;
        o_cv = o;
        if (kind != kSDown) o += (unsigned)kSKA * vec;
        total = o;
    }
    __host__ __device__ unsigned reg() const { return 16; }
    __host__ __device__ unsigned str() const { return o_str; }
    __host__ __device__ unsigned pred() const { return o_pred; }
    __host__ __device__ unsigned ro() const { return o_ro; }
    __host__ __device__ unsigned rp() const { return o_rp; }
    __host__ __device__ unsigned cv() const { return o_cv; }
};

// The two quantised arena formats: 16-bit (store.rs: i16 regrets, u16
// strategy sums) and FP8 E4M3 (both signed 8-bit), each with a per-node scale
// = the block's max magnitude, stored as value * (kR or kS) / scale.
template <int FMT>
struct QT {
    using R = int16_t;
    using S = uint16_t;
    static constexpr float kR = 32767.0f, kS = 65535.0f;
    __device__ static float dr(R q) { return (float)q; }
    __device__ static float ds(S q) { return (float)q; }
    __device__ static R er(float x) { return sat_i16(x); }
    __device__ static S es(float x) { return sat_u16(x); }
};
template <>
struct QT<kDevFP8> {
    using R = uint8_t;
    using S = uint8_t;
    static constexpr float kR = 448.0f, kS = 448.0f;
    __device__ static float dr(R q) { return e4m3_to_f32(q); }
    __device__ static float ds(S q) { return e4m3_to_f32(q); }
    __device__ static R er(float x) { return f32_to_e4m3(x); }
    __device__ static S es(float x) { return f32_to_e4m3(x); }
};
__host__ __device__ constexpr int fmt_bytes(int fmt) { return fmt == kDevF32 ? 4 : fmt == kDevFP8 ? 1 : 2; }

// Down sweep, one node per CTA: staged sigma source and parent reach; child
// reach vectors written with coalesced stores (cfr.rs:469-531 push-down).
template <int FMT, int NA, int NT = kSThreads>
__device__ __forceinline__ void ks_down_node(const Dev& d, const Arenas& ar, const SNode& it, int mode,
                                             unsigned char* sm, int& s_flag) {
    const int a = (int)it.actor, nh = d.nh[a];
    constexpr int na = NA;  // the node's action count, a compile-time constant in this instance
    const int esz = fmt_bytes(FMT);
    const SLayout L(d.nh_pad, esz, ar.pred[0] != nullptr, kSDown);
    uint64_t* bar = (uint64_t*)sm;
    unsigned char* b_reg = sm + L.reg();
    unsigned char* b_str = sm + L.str();
    unsigned char* b_pred = sm + L.pred();
    float* pr = (float*)(sm + L.ro());
    const bool has_pred = ar.pred[a] != nullptr;
    const unsigned blk = round16((unsigned)(na * nh * esz));
    if (threadIdx.x == 0) {
        // the sigma source is staged before the lock table is read (a locked
        // node's block is staged and not used)
        mbar_init(bar, 1);
        const bool u_reg = mode == 0, u_pred = u_reg && has_pred, u_str = mode != 0;
        const unsigned char* g_reg = (const unsigned char*)ar.reg[a] + it.aoff * esz;
        const unsigned char* g_str = (const unsigned char*)ar.str[a] + it.aoff * esz;
        const unsigned char* g_pred = u_pred ? (const unsigned char*)ar.pred[a] + it.aoff * esz : nullptr;
        const float* g_pr = d.reach[a] + (size_t)it.rslot * d.rstr[a];
        const unsigned vb = round16((unsigned)nh * 4u);
        s_flag = ((uintptr_t)g_reg | (uintptr_t)g_str | (uintptr_t)g_pred | (uintptr_t)g_pr) & 15u ? 1 : 0;
        if (s_flag) {
            atomicOr(d.err, 2u);
        } else {
            mbar_expect_tx(bar, (u_reg ? blk : 0u) + (u_pred ? blk : 0u) + (u_str ? blk : 0u) + vb);
            if (u_reg) bulk_load(b_reg, g_reg, blk, bar);
            if (u_pred) bulk_load(b_pred, g_pred, blk, bar);
            if (u_str) bulk_load(b_str, g_str, blk, bar);
            bulk_load(pr, g_pr, vb, bar);
        }
    }
    const long long loff = d.lock_off[a][it.sidx];
    float kr = 0.0f, kp = 0.0f;
    if (FMT != kDevF32 && mode == 0 && loff < 0) {
        kr = ar.rscale[a][it.sidx] / QT<FMT>::kR;
        if (has_pred) kp = ar.pscale[a][it.sidx] / QT<FMT>::kR;
    }
    if (!wait_staged(d, bar, &s_flag)) return;
    float sig[kSKA];
    for (int i = threadIdx.x; i < nh; i += NT) {
        s_node_sigma<FMT>(d, loff, a, i, mode, b_reg, has_pred ? b_pred : nullptr, b_str, kr, kp, na, sig);
        const float p = pr[i];
#pragma unroll
        for (int k = 0; k < kSKA; k++)
            if (k < na && it.rs[k] != kNoSlot) d.reach[a][(size_t)it.rs[k] * d.rstr[a] + i] = p * sig[k];
    }
}
template <int FMT>
__global__ void __launch_bounds__(kSThreads) ks_down(Dev d, Arenas ar, const SNode* nodes, int mode) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ int s_flag;
    const SNode it = nodes[blockIdx.x];
    switch (it.na) {  // uniform per CTA: one specialised body per action count
        case 1: ks_down_node<FMT, 1>(d, ar, it, mode, sm, s_flag); break;
        case 2: ks_down_node<FMT, 2>(d, ar, it, mode, sm, s_flag); break;
        case 3: ks_down_node<FMT, 3>(d, ar, it, mode, sm, s_flag); break;
        default: ks_down_node<FMT, 4>(d, ar, it, mode, sm, s_flag); break;
    }
}

// Up sweep, one node per CTA (cfr.rs:469-531 pull-up, 297-409 update;
// best_response.rs:69-121, 185-219 for EVAL = 1 with mode 0 BR / 1 average).
// The node's fold child, if any, is evaluated here from the staged opponent
// reach; every other child's cfv is staged from its slot.
template <int NT = kSThreads>
struct UpSharedT {  // static shared memory of ks_up (NT threads)
    int flag;
    long long S[52];
    long long dred[NT / 32];
    float red[3 * (NT / 32)];
};
using UpShared = UpSharedT<>;
// The traverser's node once its children's values are staged (cv, row k at
// cv + k * vstride) and, for the update, its regret / strategy-sum /
// prediction blocks (b_reg, b_str, b_pred) and own reach (rp): a locked
// node's value, an evaluation sweep's value (best response or average), or
// the CFR update (cfr.rs:297-409) with the blocks and scales written back.
// The node's value per hand goes to out[i] (added to it when acc_out).
__device__ __forceinline__ void s_put(float* out, int i, float v, bool add) {
    if (add) out[i] += v;
    else out[i] = v;
}
template <int FMT, int EVAL, int NA, int NT>
__device__ __forceinline__ void s_mine_node(const Dev& d, const Arenas& ar, int p, int mode, long long loff, float kr,
                                            float kp, float sscale, uint32_t sidx, uint64_t aoff, bool use_pred,
                                            unsigned char* b_reg, unsigned char* b_str, unsigned char* b_pred,
                                            float* cv, int vstride, const float* rp, float* out, bool acc_out,
                                            float* s_red) {
    const int nh = d.nh[p];
    constexpr int na = NA;
    const int esz = fmt_bytes(FMT);
    const unsigned blk = round16((unsigned)(na * nh * esz));
    float sig[kSKA];
#define CHILD_V(k, i) (cv[(k) * vstride + (i)])
    if (loff >= 0) {  // locked: fixed sigma, no update
        for (int i = threadIdx.x; i < nh; i += NT) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) acc += d.lock_sig[loff + (long long)k * nh + i] * CHILD_V(k, i);
            s_put(out, i, acc, acc_out);
        }
        return;
    }
    if (EVAL) {
        for (int i = threadIdx.x; i < nh; i += NT) {
            float acc;
            if (mode == 0) {
                acc = CHILD_V(0, i);
#pragma unroll
                for (int k = 1; k < kSKA; k++)
                    if (k < na) {
                        const float v = CHILD_V(k, i);
                        if (v > acc) acc = v;
                    }
            } else {
                s_average_sigma<FMT>(b_str, na, i, sig);
                acc = 0.0f;
#pragma unroll
                for (int k = 0; k < kSKA; k++)
                    if (k < na) acc += sig[k] * CHILD_V(k, i);
            }
            s_put(out, i, acc, acc_out);
        }
        return;
    }
    const float pos = d.disc[0], neg = d.disc[1], ds = d.disc[2];
    const void* predp = use_pred ? b_pred : nullptr;
    float v[kSKA];
    if (FMT == kDevF32) {
        float* R = (float*)b_reg;
        float* Sg = (float*)b_str;
        float* PR = (float*)b_pred;
        for (int i = threadIdx.x; i < nh; i += NT) {
            s_regret_sigma<FMT>(b_reg, predp, 0.0f, 0.0f, na, i, sig);
            float o_ = 0.0f;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) {
                    v[k] = CHILD_V(k, i);
                    o_ += sig[k] * v[k];
                }
            const float r_p = rp[i];
            const int b = i * na;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) {
                    const float r = R[b + k];
                    R[b + k] = r * (r > 0.0f ? pos : neg) + (v[k] - o_);
                    Sg[b + k] = Sg[b + k] * ds + r_p * sig[k];
                    if (use_pred) PR[b + k] = v[k] - o_;
                }
            s_put(out, i, o_, acc_out);
        }
        __syncthreads();
        store_block((unsigned char*)ar.reg[p] + aoff * esz, b_reg, blk);
        store_block((unsigned char*)ar.str[p] + aoff * esz, b_str, blk);
        if (use_pred) store_block((unsigned char*)ar.pred[p] + aoff * esz, b_pred, blk);
        return;
    }
    // Quantised arenas (cfr.rs:350-407): 16-bit, or FP8 with the same steps.
    using Q = QT<FMT == kDevFP8 ? kDevFP8 : kDevI16>;
    const float kss = sscale / Q::kS * ds;
    float rmax = 0.0f, smax = 0.0f, pmax = 0.0f;
    const bool one_pass = FMT == kDevI16 && !use_pred;
    if (one_pass) {
        int16_t* RQ = (int16_t*)b_reg;
        uint16_t* SQ = (uint16_t*)b_str;
        // Pass 1 computes every entry's new regret and strategy sum and the
        // node's maxima, keeping the f32 values in place of what it consumed:
        // the new regret where the child's value was, the new strategy sum's
        // bits split over the entry's two old 16-bit quants (each entry is
        // read and rewritten by the thread that owns its hand).  Pass 2 only
        // requantises.
        uint16_t* SQ_lo = (uint16_t*)b_reg;
        for (int i = threadIdx.x; i < nh; i += NT) {
            s_regret_sigma<FMT>(b_reg, nullptr, kr, kp, na, i, sig);
            float o_ = 0.0f;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) {
                    v[k] = CHILD_V(k, i);
                    o_ += sig[k] * v[k];
                }
            const float r_p = rp[i];
            const int b = i * na;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) {
                    const int16_t qv = RQ[b + k];
                    const float nr = (float)qv * kr * (qv > 0 ? pos : neg) + (v[k] - o_);
                    const float ns = (float)SQ[b + k] * kss + r_p * sig[k];
                    rmax = fmaxf(rmax, fabsf(nr));
                    smax = fmaxf(smax, ns);
                    cv[k * vstride + i] = nr;
                    const uint32_t bits = __float_as_uint(ns);
                    SQ_lo[b + k] = (uint16_t)(bits & 0xFFFFu);
                    SQ[b + k] = (uint16_t)(bits >> 16);
                }
            s_put(out, i, o_, acc_out);
        }
        s_block_max3<NT>(rmax, smax, pmax, s_red);
        const float rk = (rmax > 0.0f && isfinite(rmax)) ? 32767.0f / rmax : 0.0f;
        const float sk = (smax > 0.0f && isfinite(smax)) ? 65535.0f / smax : 0.0f;
        const uint32_t sr_b = ar.sr ? sr_base(d.node_id[p][sidx], *d.iter) : 0u;
        for (int i = threadIdx.x; i < nh; i += NT) {
            const int b = i * na;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) {
                    const float nr = cv[k * vstride + i];
                    const float ns = __uint_as_float((uint32_t)SQ_lo[b + k] | ((uint32_t)SQ[b + k] << 16));
                    requant16(nr, ns, rk, sk, ar.sr, sr_b, i, k, &RQ[b + k], &SQ[b + k]);
                }
        }
    }
    // Otherwise (PCFR+ predictions, or FP8, whose quants leave no room for
    // the f32 values): pass 1 finds the maxima, pass 2 recomputes from the
    // unchanged staged quants and requantises in place.
    typename Q::R* RQ = (typename Q::R*)b_reg;
    typename Q::S* SQ = (typename Q::S*)b_str;
    typename Q::R* PQ = (typename Q::R*)b_pred;
    const uint32_t sr_b2 = ar.sr && !one_pass ? sr_base(d.node_id[p][sidx], *d.iter) : 0u;
    for (int pass = one_pass ? 2 : 0; pass < 2; pass++) {
        float rk = 0.0f, sk = 0.0f, pk = 0.0f;
        if (pass == 1) {
            s_block_max3<NT>(rmax, smax, pmax, s_red);
            rk = (rmax > 0.0f && isfinite(rmax)) ? Q::kR / rmax : 0.0f;
            sk = (smax > 0.0f && isfinite(smax)) ? Q::kS / smax : 0.0f;
            pk = (pmax > 0.0f && isfinite(pmax)) ? Q::kR / pmax : 0.0f;
        }
        for (int i = threadIdx.x; i < nh; i += NT) {
            s_regret_sigma<FMT>(b_reg, predp, kr, kp, na, i, sig);
            float o_ = 0.0f;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) {
                    v[k] = CHILD_V(k, i);
                    o_ += sig[k] * v[k];
                }
            const float r_p = rp[i];
            const int b = i * na;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) {
                    const float dv = Q::dr(RQ[b + k]);  // the discount follows the stored sign
                    const float nr = dv * kr * (dv > 0.0f ? pos : neg) + (v[k] - o_);
                    const float ns = Q::ds(SQ[b + k]) * kss + r_p * sig[k];
                    if (pass == 0) {
                        rmax = fmaxf(rmax, fabsf(nr));
                        smax = fmaxf(smax, ns);
                        if (use_pred) pmax = fmaxf(pmax, fabsf(v[k] - o_));
                    } else {
                        if (FMT == kDevI16) {
                            requant16(nr, ns, rk, sk, ar.sr, sr_b2, i, k, (int16_t*)&RQ[b + k],
                                      (uint16_t*)&SQ[b + k]);
                        } else {
                            RQ[b + k] = rk > 0.0f ? Q::er(nr * rk) : (typename Q::R)0;
                            SQ[b + k] = sk > 0.0f ? Q::es(fmaxf(ns, 0.0f) * sk) : (typename Q::S)0;
                        }
                        if (use_pred) PQ[b + k] = pk > 0.0f ? Q::er((v[k] - o_) * pk) : (typename Q::R)0;
                    }
                }
            if (pass == 1) s_put(out, i, o_, acc_out);
        }
    }
#undef CHILD_V
    __syncthreads();
    store_block((unsigned char*)ar.reg[p] + aoff * esz, b_reg, blk);
    store_block((unsigned char*)ar.str[p] + aoff * esz, b_str, blk);
    if (use_pred) store_block((unsigned char*)ar.pred[p] + aoff * esz, b_pred, blk);
    if (threadIdx.x == 0) {
        ar.rscale[p][sidx] = (rmax > 0.0f && isfinite(rmax)) ? rmax : 0.0f;
        ar.sscale[p][sidx] = (smax > 0.0f && isfinite(smax)) ? smax : 0.0f;
        if (use_pred) ar.pscale[p][sidx] = (pmax > 0.0f && isfinite(pmax)) ? pmax : 0.0f;
    }
}
template <int FMT, int EVAL, int NA, bool MINE, int NT = kSThreads>
__device__ __forceinline__ void ks_up_node(const Dev& d, const Arenas& ar, const SNode& it, int p, int mode,
                                           unsigned char* sm, UpSharedT<NT>& us) {
    int& s_flag = us.flag;
    long long* s_S = us.S;
    long long* s_dred = us.dred;
    float* s_red = us.red;
    const int a = (int)it.actor, o = 1 - p, nh = d.nh[p], nho = d.nh[o];
    constexpr int na = NA;  // the node's action count, a compile-time constant in this instance
    const int esz = fmt_bytes(FMT);
    const SLayout L(d.nh_pad, esz, ar.pred[0] != nullptr, MINE ? kSUpMine : kSUpOpp);
    uint64_t* bar = (uint64_t*)sm;
    unsigned char* b_reg = sm + L.reg();
    unsigned char* b_str = sm + L.str();
    unsigned char* b_pred = sm + L.pred();
    float* ro = (float*)(sm + L.ro());
    float* rp = (float*)(sm + L.rp());
    float* cv = (float*)(sm + L.cv());
    const int vstride = d.nh_pad;
    const int fk = it.fk == kNoSlot ? -1 : (int)it.fk;
    const float famount = (int)it.folder == p ? it.tlose : it.twin;
    constexpr bool mine = MINE;  // a launch holds one actor's nodes: a == p iff MINE
    const bool has_pred = ar.pred[a] != nullptr;
    // what the node reads (an opponent node's fold child comes with the
    // folding player's reach, written by the down sweep: no strategy needed).
    // The blocks are staged before the lock table is read; a locked node's
    // are staged and not used.
    const bool use_reg = !EVAL && mine;
    const bool use_str = EVAL ? (mine && mode == 1) : mine;
    const bool use_pred = use_reg && has_pred;
    const bool use_rp = mine && !EVAL;
    const unsigned blk = round16((unsigned)(na * d.nh[a] * esz));
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        const unsigned vb = round16((unsigned)nh * 4u), vbo = round16((unsigned)nho * 4u);
        const unsigned char* g_reg = (const unsigned char*)ar.reg[a] + it.aoff * esz;
        const unsigned char* g_str = (const unsigned char*)ar.str[a] + it.aoff * esz;
        const unsigned char* g_pred = use_pred ? (const unsigned char*)ar.pred[a] + it.aoff * esz : nullptr;
        const float* g_rp = d.reach[p] + (size_t)it.rslot * d.rstr[p];
        const float* g_ro = d.reach[o] + (size_t)(mine ? it.oslot : it.rs[fk >= 0 ? fk : 0]) * d.rstr[o];
        unsigned total = (use_reg ? blk : 0u) + (use_str ? blk : 0u) + (use_pred ? blk : 0u) + (use_rp ? vb : 0u) +
                         (fk >= 0 ? vbo : 0u);
        uintptr_t bad = (uintptr_t)g_reg | (uintptr_t)g_str | (uintptr_t)g_pred;
        if (use_rp) bad |= (uintptr_t)g_rp;
        if (fk >= 0) bad |= (uintptr_t)g_ro;
#pragma unroll
        for (int k = 0; k < kSKA; k++)
            if (k < na && k != fk) {
                total += vb;
                bad |= (uintptr_t)(d.cfv + (size_t)it.cs[k] * d.nh_max);
            }
        s_flag = (bad & 15u) ? 1 : 0;
        if (s_flag) {
            atomicOr(d.err, 2u);
        } else {
            mbar_expect_tx(bar, total);
            if (use_reg) bulk_load(b_reg, g_reg, blk, bar);
            if (use_str) bulk_load(b_str, g_str, blk, bar);
            if (use_pred) bulk_load(b_pred, g_pred, blk, bar);
            if (use_rp) bulk_load(rp, g_rp, vb, bar);
            if (fk >= 0) bulk_load(ro, g_ro, vbo, bar);
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na && k != fk) bulk_load(cv + k * vstride, d.cfv + (size_t)it.cs[k] * d.nh_max, vb, bar);
        }
    }
    // lock and scales of the actor's node (16-bit arenas), loaded while the
    // copies fly
    const long long loff = d.lock_off[a][it.sidx];
    float kr = 0.0f, kp = 0.0f, sscale = 0.0f;
    if (FMT != kDevF32 && loff < 0 && mine) {
        kr = ar.rscale[a][it.sidx] / QT<FMT>::kR;
        if (has_pred) kp = ar.pscale[a][it.sidx] / QT<FMT>::kR;
        sscale = ar.sscale[a][it.sidx];
    }
    if (!wait_staged(d, bar, &s_flag)) return;

    long long ftotal = 0;
    if (fk >= 0) {
        int fsc;
        ftotal = s_fold_sums<NT>(d, o, ro, s_S, s_dred, &fsc);
        // the fold child's values go where a staged child's cfv would be
        // (fold_value of cfr_kernels.cuh with the hand's cards and same combo
        // packed in one word)
        for (int i = threadIdx.x; i < nh; i += NT) {
            const uint32_t h = d.hinfo[p][i];
            const uint32_t sm_ = h >> 16;
            const float same_r = sm_ != 0xFFFFu ? ro[sm_] : 0.0f;
            cv[fk * vstride + i] = famount * (fix_f(ftotal - s_S[h & 63u] - s_S[(h >> 6) & 63u], fsc) + same_r);
        }
        __syncthreads();
    }
    float* out = d.cfv + (size_t)it.cslot * d.nh_max;
#define CHILD_V(k, i) (cv[(k) * vstride + (i)])
    if (!mine) {  // opponent node: sum of children
        for (int i = threadIdx.x; i < nh; i += NT) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < kSKA; k++)
                if (k < na) acc += CHILD_V(k, i);
            out[i] = acc;
        }
        return;
    }
    s_mine_node<FMT, EVAL, NA, NT>(d, ar, p, mode, loff, kr, kp, sscale, it.sidx, it.aoff, use_pred, b_reg,
                                           b_str, b_pred, cv, vstride, rp, out, false, s_red);
#undef CHILD_V
}
// MINE: the launch's nodes are the traverser's (the update), else the
// opponent's (sum of children); a launch never mixes the two.
template <int FMT, int EVAL, bool MINE>
__global__ void __launch_bounds__(kSThreads) ks_up(Dev d, Arenas ar, const SNode* nodes, int p, int mode) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ UpShared us;
    const SNode it = nodes[blockIdx.x];
    switch (it.na) {  // uniform per CTA: one specialised body per action count
        case 1: ks_up_node<FMT, EVAL, 1, MINE>(d, ar, it, p, mode, sm, us); break;
        case 2: ks_up_node<FMT, EVAL, 2, MINE>(d, ar, it, p, mode, sm, us); break;
        case 3: ks_up_node<FMT, EVAL, 3, MINE>(d, ar, it, p, mode, sm, us); break;
        default: ks_up_node<FMT, EVAL, 4, MINE>(d, ar, it, p, mode, sm, us); break;
    }
}

// ------------------------------------------------- batched showdowns
// One CTA per batch of up to kShowBatch showdowns of one level that share a
// river slot (game.rs:501-577 with the plan's rank tables).  The slot's
// tables go to shared memory once per batch -- one word per scan entry (the
// opponent hands in strength order, then the 52 card lists, each the board's
// opponent hands holding the card in strength order) with the entry's hand,
// segment start and output index -- and the showdowns' opponent reach
// vectors stream through two double-buffered bulk-copy stages, two
// showdowns at a time.
//
// Per pair, with exact sums (cfr_kernels.cuh):
//   1. the two vectors' grid scales (block max);
//   2. ONE segmented scan over the concatenation [strength order (m entries)
//      | card lists (2m entries)], every thread taking a contiguous chunk:
//      a serial scan of its chunk, a shuffle scan of the chunks' (segment
//      seen, sum) pairs, the warps' carries through shared memory, and a
//      pass adding the carry to the chunk's entries before its first segment
//      start.  Output U: U[k] = reach of the k weakest opponent hands (k in
//      0..m), then card c's prefixes at msort + 1 + qbase(c) + j (the
//      layout the rank entries index);
//   3. per hand of mine, its rank entry's eight prefix values.
// Every thread works in every phase, with four block barriers per pair.
struct ShowTab {  // one slot's tables: shared-memory copies, or HBM for the last three
    const uint32_t* coff;   // 53 card-list offsets relative to the slot's first entry
    const uint32_t* ent;    // per scan entry: opponent hand | segment start << 12 | output index << 16
    const RankEntry* rank;  // mp entries (global, L1-resident across the batch)
    const uint16_t* zero;   // nz blocked traverser hands (global)
    const uint32_t* same;   // traverser same-combo map, nh entries (global)
    int m, ne, mp, nz;
};
struct ShowTabLayout {  // byte offsets of the tables inside the table region
    unsigned coff, ent, total;
};
__host__ __device__ inline unsigned r16u(unsigned b) { return (b + 15u) & ~15u; }
__host__ __device__ inline ShowTabLayout show_tab_layout(int nh_pad) {
    ShowTabLayout L;
    unsigned o = 0;
    L.coff = o;
    o += r16u(53u * 4u);
    L.ent = o;
    o += r16u(12u * nh_pad);  // 3m entries of 4 bytes (m <= nh_pad)
    L.total = o;
    return L;
}

// Slot tables of a batch into shared memory (all threads of the CTA).  The
// scan input is the concatenation [opponent hands in strength order (m) |
// card lists (ne = 2m)]; entry f's output index in U is f + 1 in the first
// part and msort + 2 + t + c for entry t of card c's list.
__device__ void load_show_tab(const Dev& d, int p, uint32_t slot, int msort, unsigned char* tabs,
                              const ShowTabLayout& TL, ShowTab& tb) {
    const int o = 1 - p;
    tb.m = (int)d.sorted_cnt[o][slot];
    const uint32_t* coff_g = d.ccard_off[o] + (size_t)slot * 53;
    const uint32_t c0 = coff_g[0];
    tb.ne = (int)(coff_g[52] - c0);
    tb.mp = (int)d.rank_cnt[p][slot];
    const uint32_t z0 = d.zero_off[p][slot];
    tb.nz = (int)(d.zero_off[p][slot + 1] - z0);
    uint32_t* t_coff = (uint32_t*)(tabs + TL.coff);
    uint32_t* t_ent = (uint32_t*)(tabs + TL.ent);
    const uint16_t* g_sidx = d.sorted_idx[o] + d.sorted_off[o][slot];
    if (threadIdx.x < 53) t_coff[threadIdx.x] = coff_g[threadIdx.x] - c0;
    const uint16_t* g_pos = d.ccard_pos[o] + c0;
    const uint8_t* g_card = d.ccard_card[o] + c0;
    const int m = tb.m, F = m + tb.ne;
    for (int f = threadIdx.x; f < F; f += blockDim.x) {
        uint32_t h, head, oi;
        if (f < m) {
            h = g_sidx[f];
            head = f == 0;
            oi = (uint32_t)f + 1u;
        } else {
            const int t = f - m;
            const uint32_t c = g_card[t];
            h = g_sidx[g_pos[t]];
            head = t == 0 || g_card[t - 1] != c;
            oi = (uint32_t)msort + 2u + (uint32_t)t + c;
        }
        t_ent[f] = h | head << 12 | oi << 16;
    }
    tb.coff = t_coff;
    tb.ent = t_ent;
    // read in place (L1-resident across the batch): keeps the CTA's shared
    // memory small, so more batches run per SM
    tb.rank = d.rank[p] + d.rank_off[p][slot];
    tb.zero = d.zero_idx[p] + z0;
    tb.same = d.same[p];
}

// Showdown CTAs have NT threads: 256 for large hand lists, 128 for small ones.
template <int NT>
__device__ void cta_showdown2(const ShowTab& tb, int nho, int msort, const float* roA, const float* roB,
                              const ShowItem& ia, const ShowItem& ib, float* outA, float* outB, longlong2* U,
                              longlong2* s_w, int* s_wf, float2* s_mx) {
    constexpr int kW = NT / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m = tb.m;
    // 1. grid scales of the two vectors
    float mxA = 0.0f, mxB = 0.0f;
    for (int j = tid; j < nho; j += NT) {
        mxA = fmaxf(mxA, roA[j]);
        mxB = fmaxf(mxB, roB[j]);
    }
    mxA = warp_max(mxA);
    mxB = warp_max(mxB);
    if (lane == 0) s_mx[warp] = make_float2(mxA, mxB);
    __syncthreads();
    mxA = s_mx[0].x;
    mxB = s_mx[0].y;
#pragma unroll
    for (int k = 1; k < kW; k++) {
        mxA = fmaxf(mxA, s_mx[k].x);
        mxB = fmaxf(mxB, s_mx[k].y);
    }
    const int scA = fix_scale(mxA), scB = fix_scale(mxB);
    // 2. segmented scan, chunk [f0, f1) per thread; an odd chunk length puts
    // the lanes' runs in distinct shared-memory banks
    const int F = m + tb.ne;
    const int chunk = ((F + NT - 1) / NT) | 1;
    const int f0 = min(tid * chunk, F), f1 = min(f0 + chunk, F);
    long long ax = 0, ay = 0;
    bool seen = false;
    for (int f = f0; f < f1; f++) {
        const uint32_t en = tb.ent[f];
        const int h = (int)(en & 0xFFFu), oi = (int)(en >> 16);
        const bool head = (en >> 12) & 1u;
        if (head) {
            ax = 0;
            ay = 0;
            seen = true;
        }
        ax += fix_q(roA[h], scA);
        ay += fix_q(roB[h], scB);
        U[oi] = make_longlong2(ax, ay);
    }
    if (tid == 0) U[0] = make_longlong2(0, 0);
    if (tid < 52) U[msort + 1 + tb.coff[tid] + tid] = make_longlong2(0, 0);
    bool fl = seen;
    long long sx = ax, sy = ay;
#pragma unroll
    for (int x = 1; x < 32; x <<= 1) {
        const int fu = __shfl_up_sync(0xffffffffu, (int)fl, x);
        const long long ux = __shfl_up_sync(0xffffffffu, sx, x);
        const long long uy = __shfl_up_sync(0xffffffffu, sy, x);
        if (lane >= x) {
            if (!fl) {
                sx += ux;
                sy += uy;
            }
            fl = fl || fu;
        }
    }
    int ef = __shfl_up_sync(0xffffffffu, (int)fl, 1);
    long long ex = __shfl_up_sync(0xffffffffu, sx, 1), ey = __shfl_up_sync(0xffffffffu, sy, 1);
    if (lane == 0) {
        ef = 0;
        ex = 0;
        ey = 0;
    }
    if (lane == 31) {
        s_w[warp] = make_longlong2(sx, sy);
        s_wf[warp] = (int)fl;
    }
    __syncthreads();
    long long cx = 0, cy = 0;
    for (int k = 0; k < warp; k++) {
        if (s_wf[k]) {
            cx = s_w[k].x;
            cy = s_w[k].y;
        } else {
            cx += s_w[k].x;
            cy += s_w[k].y;
        }
    }
    if (ef) {
        cx = ex;
        cy = ey;
    } else {
        cx += ex;
        cy += ey;
    }
    if (cx | cy) {
        for (int f = f0; f < f1; f++) {
            const uint32_t en = tb.ent[f];
            if ((en >> 12) & 1u) break;
            const int oi = (int)(en >> 16);
            longlong2 v = U[oi];
            v.x += cx;
            v.y += cy;
            U[oi] = v;
        }
    }
    __syncthreads();
    // 3. the rank entries of my hands
    const longlong2 total = U[m];
    const longlong2* Q = U + msort + 1;
    for (int k = tid; k < tb.mp; k += NT) {
        const RankEntry e = tb.rank[k];
        const int a1 = e.cards & 0xFF, a2 = e.cards >> 8;
        const longlong2 plb = U[e.lb], pub = U[e.ub], q1lo = Q[e.q1lo], q2lo = Q[e.q2lo], q1hi = Q[e.q1hi],
                        q2hi = Q[e.q2hi], s1 = Q[tb.coff[a1 + 1] + a1], s2 = Q[tb.coff[a2 + 1] + a2];
        const uint32_t sm = tb.same[e.idx];
        {
            const float lower = fix_f(plb.x - q1lo.x - q2lo.x, scA);
            const float higher = fix_f((total.x - pub.x) - (s1.x - q1hi.x) - (s2.x - q2hi.x), scA);
            const float same_r = sm != kSentinel ? roA[sm] : 0.0f;
            const float valid = fix_f(total.x - s1.x - s2.x, scA) + same_r;
            const float tied = valid - lower - higher;
            outA[e.idx] = ia.twin * lower + ia.tlose * higher + ia.ttie * tied;
        }
        if (outB) {
            const float lower = fix_f(plb.y - q1lo.y - q2lo.y, scB);
            const float higher = fix_f((total.y - pub.y) - (s1.y - q1hi.y) - (s2.y - q2hi.y), scB);
            const float same_r = sm != kSentinel ? roB[sm] : 0.0f;
            const float valid = fix_f(total.y - s1.y - s2.y, scB) + same_r;
            const float tied = valid - lower - higher;
            outB[e.idx] = ib.twin * lower + ib.tlose * higher + ib.ttie * tied;
        }
    }
    for (int z = tid; z < tb.nz; z += NT) {
        outA[tb.zero[z]] = 0.0f;
        if (outB) outB[tb.zero[z]] = 0.0f;
    }
    __syncthreads();
}
// Shared memory of ks_show_pair: two barriers, four reach buffers (two
// stages of a pair), the prefix array U (3 msort + 53 pairs), then the slot
// tables.
__host__ __device__ inline unsigned show_pair_scratch_bytes(int nh_pad, int msort) {
    return 32u + 4u * 4u * (unsigned)nh_pad + (3u * (unsigned)msort + 53u) * 16u;
}
inline size_t show_pair_smem_bytes(int nh_pad, int msort) {
    return (size_t)show_pair_scratch_bytes(nh_pad, msort) + show_tab_layout(nh_pad).total;
}
// Static shared memory of one showdown batch (NT threads).
template <int NT>
struct ShowShared {
    longlong2 w[NT / 32];
    int wf[NT / 32];
    float2 mx[NT / 32];
    int flag;
    ShowItem it[kShowBatch];
};
// One batch of showdowns (bt) on the whole CTA; sm: show_pair_smem_bytes of
// dynamic shared memory.  Returns false when a copy failed (error bits set,
// copies in flight drained).
template <int NT>
__device__ bool show_batch_run(const Dev& d, const ShowItem* items, const ShowBatch& bt, int p, int msort,
                               unsigned char* sm, ShowShared<NT>& ss) {
    int& s_flag = ss.flag;
    ShowItem* s_it = ss.it;
    const int o = 1 - p;
    const int n = (int)bt.count, npairs = (n + 1) / 2;
    uint64_t* bars = (uint64_t*)sm;
    float* rbuf = (float*)(sm + 32);
    longlong2* U = (longlong2*)(rbuf + 4 * d.nh_pad);
    unsigned char* tabs = sm + show_pair_scratch_bytes(d.nh_pad, msort);
    const ShowTabLayout TL = show_tab_layout(d.nh_pad);
    if (threadIdx.x < n) s_it[threadIdx.x] = items[bt.start + threadIdx.x];
    ShowTab tb;
    load_show_tab(d, p, bt.slot, msort, tabs, TL, tb);
    const unsigned rbytes = round16((unsigned)d.nh[o] * 4u);
    if (threadIdx.x == 0) {
        s_flag = 0;
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
    }
    __syncthreads();  // items, tables and barriers visible
    auto issue = [&](int q) {  // thread 0: pair q's reach vectors into stage q & 1
        const int st = q & 1, j0 = 2 * q, cnt = j0 + 1 < n ? 2 : 1;
        bool bad = false;
        for (int u = 0; u < cnt; u++) {
            const float* src = d.reach[o] + (size_t)s_it[j0 + u].rs[o] * d.rstr[o];
            bad = bad || ((((uintptr_t)(rbuf + (size_t)(2 * st + u) * d.nh_pad)) | (uintptr_t)src) & 15u) != 0;
        }
        if (bad) {
            s_flag = 1;
            atomicOr(d.err, 2u);
            mbar_expect_tx(&bars[st], 0);  // completes the phase with nothing in flight
            return;
        }
        mbar_expect_tx(&bars[st], rbytes * (unsigned)cnt);
        for (int u = 0; u < cnt; u++)
            bulk_load(rbuf + (size_t)(2 * st + u) * d.nh_pad, d.reach[o] + (size_t)s_it[j0 + u].rs[o] * d.rstr[o],
                      rbytes, &bars[st]);
    };
    if (threadIdx.x == 0) {
        issue(0);
        if (npairs > 1) issue(1);
    }
    for (int q = 0; q < npairs; q++) {
        const int st = q & 1;
        const bool ok = mbar_wait(&bars[st], (unsigned)(q >> 1) & 1u);
        if (__syncthreads_or(!ok) || s_flag) {
            if (threadIdx.x == 0) {
                if (!ok) atomicOr(d.err, 1u);
                // bounded drain of the copies still in flight (this pair and the next)
                mbar_wait(&bars[st], (unsigned)(q >> 1) & 1u);
                if (q + 1 < npairs) mbar_wait(&bars[st ^ 1], (unsigned)((q + 1) >> 1) & 1u);
            }
            return false;
        }
        const int j0 = 2 * q;
        const bool two = j0 + 1 < n;
        const ShowItem& ia = s_it[j0];
        const ShowItem& ib = s_it[two ? j0 + 1 : j0];
        const float* roA = rbuf + (size_t)(2 * st) * d.nh_pad;
        const float* roB = two ? roA + d.nh_pad : roA;
        cta_showdown2<NT>(tb, d.nh[o], msort, roA, roB, ia, ib, d.cfv + (size_t)ia.cslot * d.nh_max,
                          two ? d.cfv + (size_t)ib.cslot * d.nh_max : nullptr, U, ss.w, ss.wf, ss.mx);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0 && q + 2 < npairs) issue(q + 2);
    }
    return true;
}
template <int NT>
__global__ void __launch_bounds__(NT) ks_show_pair(Dev d, const ShowItem* items, const ShowBatch* batches, int p,
                                                    int msort) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ ShowShared<NT> ss;
    show_batch_run<NT>(d, items, batches[blockIdx.x], p, msort, sm, ss);
}

}  // namespace gtob
