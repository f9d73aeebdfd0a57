// Device code of the level-synchronous discounted-CFR engine (sm_100a).
//
// Kernels work on the plan's work items (host/plan.hpp).  Per-hand action
// values live in fully unrolled register arrays of KA entries (KA >= the
// widest node), so no per-hand state spills to local memory.  Terminal
// values are deterministic reductions: the plain engine accumulates them in
// f64 like the reference CPU engine (game.rs:470-577); the fused engine, which
// evaluates terminals inside their parents' kernels, accumulates in f32 like
// the reference GPU kernels (gpu/kernels.cu:117-266) to halve the shared
// memory and instruction count of the scans.
#pragma once
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "../host/solver.hpp"

namespace gtob {

enum ArenaFormatDev { kDevF32 = 0, kDevI16 = 1, kDevFP8 = 2 };

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxHpt = 6;  // hands per thread in the runout kernel (nh <= 1536)

struct Dev {
    int nh[2];
    int nh_max;        // cfv slot stride (floats, a multiple of 4: 16-byte aligned slots)
    int rstr[2];       // reach slot stride per player (floats, a multiple of 4)
    int nh_pad;        // floats per staged hand vector (multiple of 4)
    int scr_elems;     // terminal scratch elements (4 * max_sorted + 105)
    int max_nterm;     // terminal children of one action node (fused smem layout)
    const uint8_t* c1[2];
    const uint8_t* c2[2];
    const uint64_t* mask[2];
    const uint32_t* same[2];
    const float* w[2];
    const uint16_t* hperm[2];
    const uint32_t* hcard_off[2];
    const uint16_t* hcard_idx[2];
    const uint32_t* sorted_off[2];
    const uint32_t* sorted_cnt[2];
    const uint16_t* sorted_idx[2];
    const uint32_t* ccard_off[2];
    const uint16_t* ccard_pos[2];
    const uint8_t* ccard_card[2];
    const uint32_t* bin_off[2];
    const uint16_t* bin_start[2];
    const uint32_t* rank_off[2];
    const uint32_t* rank_cnt[2];
    const RankEntry* rank[2];
    const uint32_t* zero_off[2];
    const uint16_t* zero_idx[2];
    const CardEntry* cards;
    const ChildRef* crefs;
    const TermInfo* terms;
    float* reach[2];
    float* cfv;
    const long long* lock_off[2];  // per sidx, -1 = unlocked
    const float* lock_sig;
    float* disc;  // pos, neg, strat
    unsigned* iter;
    double* dot;  // root dot products
    unsigned* err;  // device error bits (bounded waits that gave up, bad copies)
    // staged engine extras
    const uint32_t* hinfo[2];   // per hand: c1 | c2 << 6 | same << 16 (0xFFFF: no same combo)
    const uint16_t* hcard52[2]; // per card: the hands holding it, 52 slots, 0xFFFF after the last
    const uint32_t* node_id[2];  // tree node id of each device action node (per player, by sidx)
    // river programs: per player o, the showdown table images of every river
    // board (river_tab_words words each) and their word offsets (num_slots + 1)
    const uint32_t* rtab[2];
    const uint32_t* rtab_off[2];
};
struct Arenas {
    void* reg[2];
    void* str[2];
    void* pred[2];  // PCFR+ only, else null
    float* rscale[2];
    float* sscale[2];
    float* pscale[2];
    int sr;  // 16-bit requantisation: 0 round to nearest even (store.rs), 1 stochastic rounding
};

// ----------------------------------------------------------- small helpers
// FP8 E4M3 arena values (the precision-study format): cvt with satfinite --
// round to nearest even, saturate to +-448 -- and the exact widening back.
__device__ __forceinline__ uint8_t f32_to_e4m3(float x) {
    return (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
}
__device__ __forceinline__ float e4m3_to_f32(uint8_t q) {
    return __half2float(__half(__nv_cvt_fp8_to_halfraw((__nv_fp8_storage_t)q, __NV_E4M3)));
}

// Rust `as i16` / `as u16` after round_ties_even (store.rs:178, 192): round to
// nearest even, saturate to the type's range, NaN -> 0.  One cvt.rni.sat each.
__device__ __forceinline__ int16_t sat_i16(float x) {
    short r;
    asm("cvt.rni.sat.s16.f32 %0, %1;" : "=h"(r) : "f"(x));
    return x != x ? (int16_t)0 : (int16_t)r;
}
__device__ __forceinline__ uint16_t sat_u16(float x) {
    unsigned short r;
    asm("cvt.rni.sat.u16.f32 %0, %1;" : "=h"(r) : "f"(x));
    return x != x ? (uint16_t)0 : (uint16_t)r;
}
// ------------------------------------------------ exact terminal sums
// Fold and showdown values need sums of opponent reach over hand subsets
// (game.rs:478-485, 512-575; the reference sums in f64 in one fixed order).
// Here the sums are exact, so any summation order gives the same bits: each
// reach value r (f32, >= 0) of one opponent vector goes on one fixed-point
// grid, q = round-half-even(r * 2^S) in an int64, with S = 51 - E for the
// vector's largest value < 2^E -- q < 2^51, and a sum of at most 1326 of
// them stays below 2^62.  Sums and differences are exact integer
// arithmetic; each difference becomes f32 once (correctly rounded, then
// scaled by 2^-S).  The grid step is 2^-51 of the vector's top power of two,
// about the rounding step of a running f64 sum.  Everything after the casts
// is the reference's f32 arithmetic.
__device__ __forceinline__ int fix_scale(float maxv) {
    const uint32_t u = __float_as_uint(maxv);
    const int e = (int)((u >> 23) & 0xFFu);
    const uint32_t m = u & 0x7FFFFFu;
    if (e == 0 && m == 0) return 0;
    const int E = e != 0 ? e - 126 : (32 - __clz((int)m)) - 149;  // maxv < 2^E
    return 51 - E;
}
__device__ __forceinline__ float pow2f(int k) { return __uint_as_float((uint32_t)(127 + k) << 23); }  // k in [-126,127]
__device__ __forceinline__ long long fix_q(float r, int S) {  // the scalings are exact
    float x = r;
    if (S > 100) {
        x = __fmul_rn(x, pow2f(100));
        S -= 100;
    }
    return __float2ll_rn(__fmul_rn(x, pow2f(S)));
}
__device__ __forceinline__ float fix_f(long long v, int S) {
    float y = __ll2float_rn(v);
    if (S > 100) {
        y = __fmul_rn(y, pow2f(-100));
        S -= 100;
    }
    return __fmul_rn(y, pow2f(-S));
}
// Accumulator types of the terminal sums: long long = the exact sums above
// (every engine), float = f32 sums like the reference GPU kernels (the
// fused32 engine).  q: one reach value onto the accumulator; f: a sum back
// to f32.  The scale argument is only used by the exact type.
template <class T>
struct Acc;
template <>
struct Acc<long long> {
    static constexpr bool kExact = true;
    __device__ static long long q(float r, int S) { return fix_q(r, S); }
    __device__ static float f(long long v, int S) { return fix_f(v, S); }
};
template <>
struct Acc<float> {
    static constexpr bool kExact = false;
    __device__ static float q(float r, int) { return r; }
    __device__ static float f(float v, int) { return v; }
};
__device__ __forceinline__ long long shfl_up_ll(long long v, int x) { return __shfl_up_sync(0xffffffffu, v, x); }

// Stochastic rounding of the 16-bit arenas' requantisation: x -> floor(x + u)
// with u in [0, 1) drawn from a hash of (tree node, iteration, hand, action),
// so the stored value is unbiased and increments below half a quantisation
// step still accumulate in expectation.  The hash is lowbias32 (Chris
// Wellons, "Hash Prospector", public domain): sr_base once per node and
// iteration, sr_bits per entry; the low 16 bits feed the regret, the high 16
// the strategy sum.  Deterministic: the oracle draws the same numbers.
__host__ __device__ __forceinline__ uint32_t lowbias32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ uint32_t sr_base(uint32_t node, uint32_t t) { return lowbias32(node ^ lowbias32(t)); }
__device__ __forceinline__ uint32_t sr_bits(uint32_t base, uint32_t hand, uint32_t action) {
    return lowbias32(base + ((hand << 4) | action) * 0x9E3779B9u);
}
__device__ __forceinline__ float sr_u_lo(uint32_t h) { return __fmul_rn((float)(h & 0xFFFFu), 0x1p-16f); }
__device__ __forceinline__ float sr_u_hi(uint32_t h) { return __fmul_rn((float)(h >> 16), 0x1p-16f); }
__device__ __forceinline__ int16_t sr_i16(float x, float u) {  // floor(x + u), saturated, NaN -> 0
    const float y = __fadd_rn(x, u);
    short r;
    asm("cvt.rmi.sat.s16.f32 %0, %1;" : "=h"(r) : "f"(y));
    return y != y ? (int16_t)0 : (int16_t)r;
}
__device__ __forceinline__ uint16_t sr_u16(float x, float u) {
    const float y = __fadd_rn(x, u);
    unsigned short r;
    asm("cvt.rmi.sat.u16.f32 %0, %1;" : "=h"(r) : "f"(y));
    return y != y ? (uint16_t)0 : (uint16_t)r;
}

// One entry's 16-bit requantisation after an update: store.rs's round to
// nearest even (sr = 0) or stochastic rounding (base = sr_base(tree node,
// iteration)).
__device__ __forceinline__ void requant16(float nr, float ns, float rk, float sk, int sr, uint32_t base, int i, int k,
                                          int16_t* rq, uint16_t* sq) {
    if (sr) {
        const uint32_t h = sr_bits(base, (uint32_t)i, (uint32_t)k);
        *rq = rk > 0.0f ? sr_i16(nr * rk, sr_u_lo(h)) : (int16_t)0;
        *sq = sk > 0.0f ? sr_u16(fmaxf(ns, 0.0f) * sk, sr_u_hi(h)) : (uint16_t)0;
    } else {
        *rq = rk > 0.0f ? sat_i16(nr * rk) : (int16_t)0;
        *sq = sk > 0.0f ? sat_u16(fmaxf(ns, 0.0f) * sk) : (uint16_t)0;
    }
}

// Block reductions of an NT-thread CTA (sh: NT / 32 entries).
template <int NT = kThreads>
__device__ __forceinline__ float block_max(float v, float* sh) {  // order-independent
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    float m = sh[0];
#pragma unroll
    for (int k = 1; k < NT / 32; k++) m = fmaxf(m, sh[k]);
    return m;
}
template <class T, int NT = kThreads>
__device__ __forceinline__ T block_sum(T v, T* sh) {  // fixed tree: deterministic
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    T s = 0;
#pragma unroll
    for (int k = 0; k < NT / 32; k++) s += sh[k];
    return s;
}

// ---------------------------------------------------- strategies of one hand
// Regret matching (cfr.rs:240-292, 875-942); entries of hand i are at
// arena[aoff + i*na + k].  Loops run over the compile-time bound KA with the
// node's na as a predicate, keeping sig[] in registers.
template <int FMT, int KA>
__device__ __forceinline__ void regret_sigma(const Arenas& ar, int actor, const ActItem& it, int i, float (&sig)[KA]) {
    const int na = (int)it.na;
    const size_t base = it.aoff + (size_t)i * na;
    float sum = 0.0f;
    if (FMT == kDevF32) {
        const float* r = (const float*)ar.reg[actor] + base;
        const float* pr = (const float*)ar.pred[actor];
#pragma unroll
        for (int k = 0; k < KA; k++)
            if (k < na) {
                float v = r[k];
                if (pr) v = fmaxf(v, 0.0f) + pr[base + k];
                sig[k] = v;
                sum += fmaxf(v, 0.0f);
            }
    } else {
        const int16_t* q = (const int16_t*)ar.reg[actor] + base;
        if (ar.pred[actor]) {
            const int16_t* qp = (const int16_t*)ar.pred[actor] + base;
            const float kr = ar.rscale[actor][it.sidx] / 32767.0f;
            const float kp = ar.pscale[actor][it.sidx] / 32767.0f;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    sig[k] = (float)max((int)q[k], 0) * kr + (float)qp[k] * kp;
                    sum += fmaxf(sig[k], 0.0f);
                }
        } else {
            int isum = 0;
            int qv[KA];
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    qv[k] = max((int)q[k], 0);
                    isum += qv[k];
                }
            if (isum > 0) {
                const float inv = 1.0f / (float)isum;
#pragma unroll
                for (int k = 0; k < KA; k++)
                    if (k < na) sig[k] = (float)qv[k] * inv;
            } else {
                const float u = 1.0f / (float)na;
#pragma unroll
                for (int k = 0; k < KA; k++)
                    if (k < na) sig[k] = u;
            }
            return;
        }
    }
    if (sum > 1e-12f) {
        const float inv = 1.0f / sum;
#pragma unroll
        for (int k = 0; k < KA; k++)
            if (k < na) sig[k] = fmaxf(sig[k], 0.0f) * inv;
    } else {
        const float u = 1.0f / (float)na;
#pragma unroll
        for (int k = 0; k < KA; k++)
            if (k < na) sig[k] = u;
    }
}
// Average strategy (cfr.rs:679-726).
template <int FMT, int KA>
__device__ __forceinline__ void average_sigma(const Arenas& ar, int actor, const ActItem& it, int i, float (&sig)[KA]) {
    const int na = (int)it.na;
    const size_t base = it.aoff + (size_t)i * na;
    if (FMT == kDevF32) {
        const float* s = (const float*)ar.str[actor] + base;
        double sum = 0.0;
        float v[KA];
#pragma unroll
        for (int k = 0; k < KA; k++)
            if (k < na) {
                v[k] = fmaxf(s[k], 0.0f);
                sum += (double)v[k];
            }
        if (sum > 1e-12) {
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) sig[k] = (float)((double)v[k] / sum);
        } else {
            const float u = 1.0f / (float)na;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) sig[k] = u;
        }
    } else {
        const uint16_t* q = (const uint16_t*)ar.str[actor] + base;
        unsigned sum = 0;
        unsigned qv[KA];
#pragma unroll
        for (int k = 0; k < KA; k++)
            if (k < na) {
                qv[k] = q[k];
                sum += qv[k];
            }
        if (sum > 0) {
            const float inv = 1.0f / (float)sum;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) sig[k] = (float)qv[k] * inv;
        } else {
            const float u = 1.0f / (float)na;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) sig[k] = u;
        }
    }
}
// The strategy an action node plays for one hand in a sweep: the lock if
// any, else regret matching (mode 0, CFR) or the average strategy (mode 1).
template <int FMT, int KA>
__device__ __forceinline__ void node_sigma(const Dev& d, const Arenas& ar, const ActItem& it, long long loff, int i,
                                           int mode, float (&sig)[KA]) {
    const int na = (int)it.na;
    if (loff >= 0) {
        const int nh = d.nh[it.actor];
#pragma unroll
        for (int k = 0; k < KA; k++)
            if (k < na) sig[k] = d.lock_sig[loff + (long long)k * nh + i];
    } else if (mode == 0) {
        regret_sigma<FMT, KA>(ar, (int)it.actor, it, i, sig);
    } else {
        average_sigma<FMT, KA>(ar, (int)it.actor, it, i, sig);
    }
}

// ------------------------------------------------------ terminal evaluators
// Fold (game.rs:470-496) in two halves so terminals sharing one opponent
// reach vector share the sums: fold_sums -> total and per-card sums S[52];
// fold_write -> out[i] = amount * ((T - S[c1] - S[c2]) + same).
// A card lies in at most 51 two-card hands, so every per-card list fits two
// 32-lane chunks.  Each warp owns kCardsPerWarp cards and issues all their
// index and reach loads before reducing, so the lists cost one round trip
// per dependent load level instead of one per card.
constexpr int kCardsPerWarp = (52 + kWarps - 1) / kWarps;

// Scale of the exact sums over one opponent reach vector (all threads of an
// NT-thread CTA; 0 for the f32 accumulator).  sh: NT / 32 floats.
template <class T, int NT = kThreads>
__device__ __forceinline__ int vec_scale(const float* ro, int n, float* sh) {
    if (!Acc<T>::kExact) return 0;
    float m = 0.0f;
    for (int j = threadIdx.x; j < n; j += blockDim.x) m = fmaxf(m, ro[j]);
    return fix_scale(block_max<NT>(m, sh));
}
template <class T>
__device__ T fold_sums(const Dev& d, int o, const float* ro, T* S, T* s_red, int& sc) {
    const int nho = d.nh[o];
    sc = vec_scale<T>(ro, nho, (float*)s_red);
    T t = 0;
#pragma unroll
    for (int u = 0; u < kMaxHpt; u++) {
        const int j = threadIdx.x + u * kThreads;
        if (j < nho) t += Acc<T>::q(ro[j], sc);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t* off = d.hcard_off[o];
    const uint16_t* idx = d.hcard_idx[o];
    T v[kCardsPerWarp][2];
#pragma unroll
    for (int ci = 0; ci < kCardsPerWarp; ci++) {
        const int c = warp + ci * kWarps;
        const uint32_t b = c < 52 ? off[c] : 0, e = c < 52 ? off[c + 1] : 0;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t k = b + lane + 32 * h;
            v[ci][h] = k < e ? Acc<T>::q(ro[idx[k]], sc) : (T)0;
        }
    }
    const T total = block_sum<T>(t, s_red);
#pragma unroll
    for (int ci = 0; ci < kCardsPerWarp; ci++) {
        T s = v[ci][0] + v[ci][1];
#pragma unroll
        for (int x = 16; x > 0; x >>= 1) s += __shfl_xor_sync(0xffffffffu, s, x);
        const int c = warp + ci * kWarps;
        if (lane == 0 && c < 52) S[c] = s;
    }
    __syncthreads();
    return total;
}
template <class T>
__device__ void fold_write(const Dev& d, int p, const float* ro, T total, const T* S, int sc, float amount,
                           float* out) {
    const int nhp = d.nh[p];
    for (int i = threadIdx.x; i < nhp; i += blockDim.x) {
        const uint32_t sm = d.same[p][i];
        const float same_r = sm != kSentinel ? ro[sm] : 0.0f;
        const float valid = Acc<T>::f(total - S[d.c1[p][i]] - S[d.c2[p][i]], sc) + same_r;
        out[i] = amount * valid;
    }
}

// Block exclusive scan of x[0..m) into out[0..m], out[m] = total (fixed
// order; an NT-thread CTA, s_w: NT / 32 entries).
template <class T, int NT = kThreads>
__device__ void block_exclusive_scan(const T* x, T* out, int m, T* s_w) {
    const int tid = threadIdx.x;
    const int chunk = (m + NT - 1) / NT;
    const int lo = min(tid * chunk, m), hi = min(lo + chunk, m);
    T local = 0;
    for (int k = lo; k < hi; k++) local += x[k];
    T incl = local;
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    T wbase = 0;
    for (int k = 0; k < warp; k++) wbase += s_w[k];
    T run = wbase + (incl - local);
    for (int k = lo; k < hi; k++) {
        out[k] = run;
        run += x[k];
    }
    if (tid == NT - 1) {
        T tot = 0;
#pragma unroll
        for (int k = 0; k < NT / 32; k++) tot += s_w[k];
        out[m] = tot;
    }
}

// Showdown (game.rs:501-577) as a strength-sorted prefix scan with
// card-removal corrections.  Scratch `sh` (4m + 105 elements): R (sorted
// opponent reach), P (exclusive prefix of R, P[m] = total), Q (per-card
// exclusive prefixes, concatenated), S (per-card totals).  My hands absent
// from the board's list get 0.  Ends with a barrier.  NT threads (s_w: NT /
// 32 entries); the exact sums make the result independent of NT.
template <class T, int NT = kThreads>
__device__ void eval_showdown(const Dev& d, int p, uint32_t slot, const float* ro, float win, float lose, float tie,
                              float* out, T* sh, T* s_w) {
    const int o = 1 - p;
    const int m = (int)d.sorted_cnt[o][slot];
    const uint16_t* sidx = d.sorted_idx[o] + d.sorted_off[o][slot];
    const uint32_t* coff = d.ccard_off[o] + (size_t)slot * 53;
    const uint16_t* cpos = d.ccard_pos[o];
    T* R = sh;
    T* P = R + m;
    T* Q = P + m + 1;
    T* S = Q + 2 * m + 52;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t c0 = coff[0];
    const int sc = vec_scale<T, NT>(ro, d.nh[o], (float*)s_w);
    if (threadIdx.x < 52) Q[(coff[threadIdx.x] - c0) + threadIdx.x] = 0;  // each card's exclusive prefix starts at 0
    for (int k = threadIdx.x; k < m; k += NT) R[k] = Acc<T>::q(ro[sidx[k]], sc);
    __syncthreads();
    block_exclusive_scan<T, NT>(R, P, m, s_w);
    // Per-card exclusive prefixes: whole card lists are packed into bins of
    // <= 64 entries (plan time), so one warp scans a bin as two 32-lane
    // chunks of a segmented scan (segments = cards) with no cross-warp carry.
    const uint16_t* bs = d.bin_start[o] + d.bin_off[o][slot];
    const int nbins = (int)(d.bin_off[o][slot + 1] - d.bin_off[o][slot]) - 1;
    const uint16_t* bpos = cpos + c0;
    const uint8_t* bcard = d.ccard_card[o] + c0;
    for (int b = warp; b < nbins; b += NT / 32) {
        const uint32_t t0 = bs[b], t1 = bs[b + 1];
        T carry = 0;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t t = t0 + 32 * h + lane;
            const bool valid = t < t1;
            const int c = valid ? bcard[t] : 255;
            const int pc = (valid && t > t0) ? bcard[t - 1] : 255;
            T s = valid ? R[bpos[t]] : (T)0;
            unsigned f = valid && pc != c;  // first entry of its card in this bin
#pragma unroll
            for (int x = 1; x < 32; x <<= 1) {
                const T y = __shfl_up_sync(0xffffffffu, s, x);
                const unsigned g = __shfl_up_sync(0xffffffffu, f, x);
                if (lane >= x) {
                    if (!f) s += y;
                    f |= g;
                }
            }
            if (!f) s += carry;  // the card continued from the previous chunk
            if (valid) Q[t + c + 1] = s;
            carry = __shfl_sync(0xffffffffu, s, 31);
        }
    }
    __syncthreads();
    if (threadIdx.x < 52) S[threadIdx.x] = Q[(coff[threadIdx.x + 1] - c0) + threadIdx.x];
    __syncthreads();
    const T total = P[m];
    const int mp = (int)d.rank_cnt[p][slot];
    const RankEntry* re = d.rank[p] + d.rank_off[p][slot];
    for (int k = threadIdx.x; k < mp; k += blockDim.x) {
        const RankEntry e = re[k];
        const int a1 = e.cards & 0xFF, a2 = e.cards >> 8;
        const float lower = Acc<T>::f(P[e.lb] - Q[e.q1lo] - Q[e.q2lo], sc);
        const float higher = Acc<T>::f((total - P[e.ub]) - (S[a1] - Q[e.q1hi]) - (S[a2] - Q[e.q2hi]), sc);
        const uint32_t sm = d.same[p][e.idx];
        const float same_r = sm != kSentinel ? ro[sm] : 0.0f;
        const float valid = Acc<T>::f(total - S[a1] - S[a2], sc) + same_r;
        const float tied = valid - lower - higher;
        out[e.idx] = win * lower + lose * higher + tie * tied;
    }
    for (uint32_t z = d.zero_off[p][slot] + threadIdx.x; z < d.zero_off[p][slot + 1]; z += blockDim.x)
        out[d.zero_idx[p][z]] = 0.0f;
    __syncthreads();
}

// ------------------------------------------------------------------ kernels
__device__ __forceinline__ void begin_iteration(unsigned* iter, float* disc, int algo) {
    // cfr.rs:44-64, in f64 on the device from the device iteration counter
    const unsigned t = ++(*iter);
    const double td = (double)t;
    const double q = td / (td + 1.0);
    if (algo == kDcfr) {
        const double ta = pow(td, 1.5);
        disc[0] = (float)(ta / (ta + 1.0));
        disc[1] = 0.5f;
    } else {
        disc[0] = 1.0f;
        disc[1] = 0.0f;
    }
    disc[2] = (float)(q * q);
}
__global__ void k_begin_iteration(unsigned* iter, float* disc, int algo) { begin_iteration(iter, disc, algo); }

__global__ void k_copy_root(Dev d) {
    for (int q = 0; q < 2; q++)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.nh[q]; i += gridDim.x * blockDim.x)
            d.reach[q][i] = d.w[q][i];
}

// Down sweep, action nodes: child actor reach = parent reach * sigma, for
// every child that keeps a reach slot.  mode 0: current strategy, 1: average.
template <int FMT, int KA>
__global__ void __launch_bounds__(kThreads) k_down_action(Dev d, Arenas ar, const ActItem* items, int mode) {
    __shared__ uint32_t s_rs[KA];
    const ActItem it = items[blockIdx.x];
    const int a = (int)it.actor, na = (int)it.na, nh = d.nh[a];
    if (threadIdx.x < na) s_rs[threadIdx.x] = d.crefs[it.cref + threadIdx.x].rslot;
    __syncthreads();
    const float* parent = d.reach[a] + (size_t)it.rslot * d.rstr[a];
    const long long loff = d.lock_off[a][it.sidx];
    float sig[KA];
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
        const float pr = parent[i];
        node_sigma<FMT, KA>(d, ar, it, loff, i, mode, sig);
#pragma unroll
        for (int k = 0; k < KA; k++)
            if (k < na && s_rs[k] != kNoSlot) d.reach[a][(size_t)s_rs[k] * d.rstr[a] + i] = pr * sig[k];
    }
}

// Down sweep, chance edges: both players' reach with holders of the card zeroed.
// qmask: the players whose reach is refreshed (bit q)
__device__ __forceinline__ void edge_down(const Dev& d, const EdgeItem& e, int qmask) {
    for (int q = 0; q < 2; q++) {
        if (!(qmask >> q & 1)) continue;
        const int nh = d.nh[q];
        const float* pr = d.reach[q] + (size_t)e.prs[q] * d.rstr[q];
        float* cr = d.reach[q] + (size_t)e.crs[q] * d.rstr[q];
        for (int i = threadIdx.x; i < nh; i += blockDim.x) cr[i] = (d.mask[q][i] >> e.card & 1ull) ? 0.0f : pr[i];
    }
}
__global__ void __launch_bounds__(kThreads) k_down_chance(Dev d, const EdgeItem* items, int qmask) {
    edge_down(d, items[blockIdx.x], qmask);
}

// Plain engine terminal kernels (exact sums): one CTA per terminal, result to its cfv slot.
__global__ void __launch_bounds__(kThreads) k_fold(Dev d, const FoldItem* items, int p) {
    __shared__ long long S[52];
    __shared__ long long s_red[kWarps];
    const FoldItem f = items[blockIdx.x];
    const int o = 1 - p;
    const float* ro = d.reach[o] + (size_t)f.rs[o] * d.rstr[o];
    int sc;
    const long long total = fold_sums<long long>(d, o, ro, S, s_red, sc);
    fold_write<long long>(d, p, ro, total, S, sc, (int)f.folder == p ? f.tlose : f.twin,
                          d.cfv + (size_t)f.cslot * d.nh_max);
}
__global__ void __launch_bounds__(kThreads) k_showdown(Dev d, const ShowItem* items, int p) {
    extern __shared__ long long sh[];
    __shared__ long long s_w[kWarps];
    const ShowItem s = items[blockIdx.x];
    const int o = 1 - p;
    const float* ro = d.reach[o] + (size_t)s.rs[o] * d.rstr[o];
    eval_showdown<long long>(d, p, s.slot, ro, s.twin, s.tlose, s.ttie, d.cfv + (size_t)s.cslot * d.nh_max, sh,
                             s_w);
}

// Chance node (cfr.rs:637-663): sum of representative children through the
// suit-permutation hand tables, skipping holders of the card, times
// 1/divisor.  All-in runout children (showdowns) are evaluated in place (T
// is the runout showdowns' accumulator type).
// (NT threads; s_w: NT / 32 entries; dsm: the runout scratch; nh <=
// kMaxHpt * kThreads, which the engine checks)
template <class T, int NT = kThreads>
__device__ void chance_node(const Dev& d, const ChanceItem& c, int p, double* dsm, T* s_w) {
    constexpr int HPT = kMaxHpt * kThreads / NT;  // hands per thread
    const int nh = d.nh[p], o = 1 - p, nho = d.nh[o];
    float* out = d.cfv + (size_t)c.cslot * d.nh_max;
    if (c.nterm == 0) {
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            const uint64_t hm = d.mask[p][i];
            float acc = 0.0f;
            for (uint32_t t = c.cc_start; t < c.cc_start + c.cc_count; t++) {
                const CardEntry e = d.cards[t];
                if (hm >> (e.card & 0xFF) & 1ull) continue;
                const int src = e.perm ? (int)d.hperm[p][(size_t)e.perm * nh + i] : i;
                acc += d.cfv[(size_t)e.child_cslot * d.nh_max + src];
            }
            out[i] = acc * c.inv;
        }
        return;
    }
    T* scr = (T*)dsm;
    float* rt = (float*)(scr + d.scr_elems);
    float* tv = rt + d.nh_pad;
    const float* ro = d.reach[o] + (size_t)c.rs[o] * d.rstr[o];
    float acc[HPT];
#pragma unroll
    for (int k = 0; k < HPT; k++) acc[k] = 0.0f;
    uint32_t have = kNoSlot;
    for (uint32_t t = c.cc_start; t < c.cc_start + c.cc_count; t++) {
        const CardEntry e = d.cards[t];
        const int card = e.card & 0xFF;
        const float* src_v;
        if (e.term != kNoSlot) {
            if (e.term != have) {
                const int rep = (e.card >> 8) & 0xFF;
                for (int j = threadIdx.x; j < nho; j += blockDim.x) rt[j] = (d.mask[o][j] >> rep & 1ull) ? 0.0f : ro[j];
                __syncthreads();
                const TermInfo tm = d.terms[e.term];
                eval_showdown<T, NT>(d, p, tm.aux, rt, tm.twin, tm.tlose, tm.ttie, tv, scr, s_w);
                have = e.term;
            }
            src_v = tv;
        } else {
            src_v = d.cfv + (size_t)e.child_cslot * d.nh_max;
        }
#pragma unroll
        for (int k = 0; k < HPT; k++) {
            const int i = threadIdx.x + k * NT;
            if (i < nh && !(d.mask[p][i] >> card & 1ull)) {
                const int src = e.perm ? (int)d.hperm[p][(size_t)e.perm * nh + i] : i;
                acc[k] += src_v[src];
            }
        }
        __syncthreads();  // tv / rt are rewritten by the next runout card
    }
#pragma unroll
    for (int k = 0; k < HPT; k++) {
        const int i = threadIdx.x + k * NT;
        if (i < nh) out[i] = acc[k] * c.inv;
    }
}
template <class T>
__global__ void __launch_bounds__(kThreads) k_chance(Dev d, const ChanceItem* items, int p) {
    extern __shared__ double dsm[];
    __shared__ T s_w[kWarps];
    chance_node<T>(d, items[blockIdx.x], p, dsm, s_w);
}

// Up sweep, action nodes.  EVAL = 0: CFR update (cfr.rs:469-531 with
// update_node 297-409).  EVAL = 1: evaluation (best_response.rs:69-121,
// 185-219), mode 0 best response, mode 1 average strategy.  Terminal
// children (fused engine, f32 sums) are evaluated first into shared memory:
// dynamic smem = [scratch: scr_elems floats][opp reach per terminal:
// max_nterm x nh_pad][terminal values: max_nterm x nh_pad].
template <int FMT, int EVAL, int KA, class TT>
__global__ void __launch_bounds__(kThreads) k_up_action(Dev d, Arenas ar, const ActItem* items, int p, int mode) {
    extern __shared__ double dsm[];
    __shared__ float s_red[kWarps];
    __shared__ TT s_redt[kWarps];
    __shared__ TT s_S[52];
    __shared__ uint32_t s_src[KA];  // cfv slot, or terminal ordinal | 0x80000000
    const ActItem it = items[blockIdx.x];
    const int a = (int)it.actor, na = (int)it.na, nh = d.nh[p], o = 1 - p, nho = d.nh[o];
    if (threadIdx.x < na) {
        const ChildRef c = d.crefs[it.cref + threadIdx.x];
        uint32_t ti = 0;
        for (int k = 0; k < (int)threadIdx.x; k++) ti += d.crefs[it.cref + k].kind != kChildNode;
        s_src[threadIdx.x] = c.kind == kChildNode ? c.cslot : (0x80000000u | ti);
    }
    __syncthreads();
    float* out = d.cfv + (size_t)it.cslot * d.nh_max;
    const size_t stride = (size_t)d.nh_max;
    const long long loff = d.lock_off[a][it.sidx];
    float sig[KA];
    float* tv = nullptr;
    if (it.nterm) {
        TT* scr = (TT*)dsm;
        float* rts = (float*)(scr + d.scr_elems);
        tv = rts + (size_t)d.max_nterm * d.nh_pad;
        const float* ro = d.reach[o] + (size_t)(a == o ? it.rslot : it.oslot) * d.rstr[o];
        if (a == o) {
            // the opponent acts: each terminal child's reach = reach * sigma_o[k]
            for (int j = threadIdx.x; j < nho; j += blockDim.x) {
                node_sigma<FMT, KA>(d, ar, it, loff, j, EVAL ? 1 : 0, sig);
                const float r = ro[j];
#pragma unroll
                for (int k = 0; k < KA; k++)
                    if (k < na && (s_src[k] & 0x80000000u))
                        rts[(size_t)(s_src[k] & 0x7FFFFFFFu) * d.nh_pad + j] = r * sig[k];
            }
            __syncthreads();
        }
        TT total = 0;
        int fsc = 0;
        bool have_sums = false;
        int t = 0;
        for (int k = 0; k < na; k++) {
            const ChildRef c = d.crefs[it.cref + k];
            if (c.kind == kChildNode) continue;
            const float* rk = a == o ? rts + (size_t)t * d.nh_pad : ro;
            const TermInfo tm = d.terms[c.term];
            float* dst = tv + (size_t)t * d.nh_pad;
            if (c.kind == kChildFold) {
                if (!have_sums) total = fold_sums<TT>(d, o, rk, s_S, s_redt, fsc);
                have_sums = a == p;  // every terminal below my own node shares one opponent reach
                fold_write<TT>(d, p, rk, total, s_S, fsc, (int)tm.aux == p ? tm.tlose : tm.twin, dst);
                __syncthreads();
            } else {
                eval_showdown<TT>(d, p, tm.aux, rk, tm.twin, tm.tlose, tm.ttie, dst, scr, s_redt);
            }
            t++;
        }
    }
#define CHILD_V(k, i) \
    (s_src[k] & 0x80000000u ? tv[(size_t)(s_src[k] & 0x7FFFFFFFu) * d.nh_pad + (i)] : d.cfv[(size_t)s_src[k] * stride + (i)])
    if (a != p) {  // opponent node: sum of children
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) acc += CHILD_V(k, i);
            out[i] = acc;
        }
        return;
    }
    if (loff >= 0) {  // locked: fixed sigma, no update, in both sweeps
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) acc += d.lock_sig[loff + (long long)k * nh + i] * CHILD_V(k, i);
            out[i] = acc;
        }
        return;
    }
    if (EVAL) {
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            float acc;
            if (mode == 0) {
                acc = CHILD_V(0, i);
#pragma unroll
                for (int k = 1; k < KA; k++)
                    if (k < na) {
                        const float v = CHILD_V(k, i);
                        if (v > acc) acc = v;
                    }
            } else {
                average_sigma<FMT, KA>(ar, a, it, i, sig);
                acc = 0.0f;
#pragma unroll
                for (int k = 0; k < KA; k++)
                    if (k < na) acc += sig[k] * CHILD_V(k, i);
            }
            out[i] = acc;
        }
        return;
    }
    const float pos = d.disc[0], neg = d.disc[1], ds = d.disc[2];
    const float* reach = d.reach[p] + (size_t)it.rslot * d.rstr[p];
    float v[KA];
    if (FMT == kDevF32) {
        float* R = (float*)ar.reg[p];
        float* S = (float*)ar.str[p];
        float* PR = (float*)ar.pred[p];
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            regret_sigma<FMT, KA>(ar, p, it, i, sig);
            float o_ = 0.0f;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    v[k] = CHILD_V(k, i);
                    o_ += sig[k] * v[k];
                }
            const float rp = reach[i];
            const size_t b = it.aoff + (size_t)i * na;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    const float r = R[b + k];
                    R[b + k] = r * (r > 0.0f ? pos : neg) + (v[k] - o_);
                    S[b + k] = S[b + k] * ds + rp * sig[k];
                    if (PR) PR[b + k] = v[k] - o_;
                }
            out[i] = o_;
        }
        return;
    }
    // 16-bit arenas: pass 1 finds the new block maxima, pass 2 recomputes and
    // requantises (cfr.rs:350-407), then the node scales are replaced.
    int16_t* RQ = (int16_t*)ar.reg[p];
    uint16_t* SQ = (uint16_t*)ar.str[p];
    int16_t* PQ = (int16_t*)ar.pred[p];
    const float kr = ar.rscale[p][it.sidx] / 32767.0f;
    const float kss = ar.sscale[p][it.sidx] / 65535.0f * ds;
    const uint32_t sr_b = ar.sr ? sr_base(it.node, *d.iter) : 0u;
    float rmax = 0.0f, smax = 0.0f, pmax = 0.0f;
    for (int pass = 0; pass < 2; pass++) {
        float rk = 0.0f, sk = 0.0f, pk = 0.0f;
        if (pass == 1) {
            rmax = block_max(rmax, s_red);
            smax = block_max(smax, s_red);
            if (PQ) pmax = block_max(pmax, s_red);
            rk = (rmax > 0.0f && isfinite(rmax)) ? 32767.0f / rmax : 0.0f;
            sk = (smax > 0.0f && isfinite(smax)) ? 65535.0f / smax : 0.0f;
            pk = (pmax > 0.0f && isfinite(pmax)) ? 32767.0f / pmax : 0.0f;
        }
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            regret_sigma<FMT, KA>(ar, p, it, i, sig);
            float o_ = 0.0f;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    v[k] = CHILD_V(k, i);
                    o_ += sig[k] * v[k];
                }
            const float rp = reach[i];
            const size_t b = it.aoff + (size_t)i * na;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    const int16_t qv = RQ[b + k];
                    const float nr = (float)qv * kr * (qv > 0 ? pos : neg) + (v[k] - o_);
                    const float ns = (float)SQ[b + k] * kss + rp * sig[k];
                    if (pass == 0) {
                        rmax = fmaxf(rmax, fabsf(nr));
                        smax = fmaxf(smax, ns);
                        if (PQ) pmax = fmaxf(pmax, fabsf(v[k] - o_));
                    } else {
                        requant16(nr, ns, rk, sk, ar.sr, sr_b, i, k, &RQ[b + k], &SQ[b + k]);
                        if (PQ) PQ[b + k] = pk > 0.0f ? sat_i16((v[k] - o_) * pk) : (int16_t)0;
                    }
                }
            if (pass == 1) out[i] = o_;
        }
    }
#undef CHILD_V
    __syncthreads();  // every thread has read the old scales
    if (threadIdx.x == 0) {
        ar.rscale[p][it.sidx] = (rmax > 0.0f && isfinite(rmax)) ? rmax : 0.0f;
        ar.sscale[p][it.sidx] = (smax > 0.0f && isfinite(smax)) ? smax : 0.0f;
        if (PQ) ar.pscale[p][it.sidx] = (pmax > 0.0f && isfinite(pmax)) ? pmax : 0.0f;
    }
}

// ------------------------------------------------- warp-per-node kernels
// The fast engine gives each action node (and each plain fold) one warp:
// eight nodes per CTA, no block barriers, a lane walks hands lane, lane+32,
// ... so a node's hands are independent and a warp never waits for another.

template <class T>
__device__ __forceinline__ T warp_sum(T v) {  // fixed xor tree: deterministic
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Fold summary of one opponent reach vector by one warp (game.rs:478-485),
// exact sums: the vector's grid scale (warp max), the total and the 52
// per-card sums (lane c and lane c + 32 each sum card c's hand list).  S: 52
// entries private to the warp.
__device__ long long warp_fold_sums(const Dev& d, int o, const float* ro, long long* S, int& sc) {
    const int lane = threadIdx.x & 31, nho = d.nh[o];
    float mx = 0.0f;
    for (int j = lane; j < nho; j += 32) mx = fmaxf(mx, ro[j]);
    sc = fix_scale(warp_max(mx));
    long long t = 0;
#pragma unroll 4
    for (int j = lane; j < nho; j += 32) t += fix_q(ro[j], sc);
#pragma unroll
    for (int cc = 0; cc < 2; cc++) {
        const int c = lane + 32 * cc;
        if (c < 52) {
            const uint32_t b = d.hcard_off[o][c], e = d.hcard_off[o][c + 1];
            long long s = 0;
#pragma unroll 4
            for (uint32_t k = b; k < e; k++) s += fix_q(ro[d.hcard_idx[o][k]], sc);
            S[c] = s;
        }
    }
    __syncwarp();
#pragma unroll
    for (int x = 16; x > 0; x >>= 1) t += __shfl_xor_sync(0xffffffffu, t, x);
    return t;
}
// One hand's fold value from the warp's summary.
__device__ __forceinline__ float fold_value(const Dev& d, int p, int i, const float* ro, long long total,
                                            const long long* S, int sc, float amount) {
    const uint32_t sm = d.same[p][i];
    const float same_r = sm != kSentinel ? ro[sm] : 0.0f;
    return amount * (fix_f(total - S[d.c1[p][i]] - S[d.c2[p][i]], sc) + same_r);
}

#define WARP_ITEM(count)                                              \
    const int wid = blockIdx.x * kWarps + (int)(threadIdx.x >> 5);   \
    if (wid >= (count)) return;                                       \
    const int lane = threadIdx.x & 31;

template <int FMT, int KA>
__global__ void __launch_bounds__(kThreads) kw_down_action(Dev d, Arenas ar, const ActItem* items, int count, int mode) {
    WARP_ITEM(count)
    const ActItem it = items[wid];
    const int a = (int)it.actor, na = (int)it.na, nh = d.nh[a];
    uint32_t rs[KA];
#pragma unroll
    for (int k = 0; k < KA; k++) rs[k] = k < na ? d.crefs[it.cref + k].rslot : kNoSlot;
    const float* parent = d.reach[a] + (size_t)it.rslot * d.rstr[a];
    float* rbase = d.reach[a];
    const long long loff = d.lock_off[a][it.sidx];
    float sig[KA];
#pragma unroll 2
    for (int i = lane; i < nh; i += 32) {
        const float pr = parent[i];
        node_sigma<FMT, KA>(d, ar, it, loff, i, mode, sig);
#pragma unroll
        for (int k = 0; k < KA; k++)
            if (k < na && rs[k] != kNoSlot) rbase[(size_t)rs[k] * d.rstr[a] + i] = pr * sig[k];
    }
}

// Plain-layout fold terminal, one warp per fold: result to its cfv slot.
__global__ void __launch_bounds__(kThreads) kw_fold(Dev d, const FoldItem* items, int count, int p) {
    __shared__ long long s_S[kWarps][52];
    WARP_ITEM(count)
    const FoldItem f = items[wid];
    const int o = 1 - p;
    const float* ro = d.reach[o] + (size_t)f.rs[o] * d.rstr[o];
    long long* S = s_S[threadIdx.x >> 5];
    int sc;
    const long long total = warp_fold_sums(d, o, ro, S, sc);
    const float amount = (int)f.folder == p ? f.tlose : f.twin;
    float* out = d.cfv + (size_t)f.cslot * d.nh_max;
    for (int i = lane; i < d.nh[p]; i += 32) out[i] = fold_value(d, p, i, ro, total, S, sc, amount);
}

// Up sweep, action nodes, one warp per node.  Fold children are evaluated in
// place from a warp fold summary (the node's single fold child, if any);
// every other child is read from its cfv slot.  EVAL = 0: CFR update
// (cfr.rs:469-531, 297-409); EVAL = 1: best response (mode 0) or average
// strategy (mode 1), best_response.rs:69-121, 185-219.  Dynamic smem per
// warp: the fold child's opponent reach when the opponent acts (nh_pad floats).
template <int FMT, int EVAL, int KA>
__global__ void __launch_bounds__(kThreads) kw_up_action(Dev d, Arenas ar, const ActItem* items, int count, int p,
                                                         int mode) {
    extern __shared__ float wsm[];
    __shared__ long long s_S[kWarps][52];
    WARP_ITEM(count)
    const int w = threadIdx.x >> 5;
    const ActItem it = items[wid];
    const int a = (int)it.actor, na = (int)it.na, nh = d.nh[p], o = 1 - p, nho = d.nh[o];
    uint32_t cs[KA];
    int fk = -1;  // the fold child, if evaluated here
    float famount = 0.0f;
#pragma unroll
    for (int k = 0; k < KA; k++) {
        cs[k] = 0;
        if (k < na) {
            const ChildRef c = d.crefs[it.cref + k];
            cs[k] = c.cslot;
            if (c.kind == kChildFold) {
                fk = k;
                const TermInfo tm = d.terms[c.term];
                famount = (int)tm.aux == p ? tm.tlose : tm.twin;
            }
        }
    }
    const long long loff = d.lock_off[a][it.sidx];
    float sig[KA];
    long long ftotal = 0;
    int fsc = 0;
    const long long* S = s_S[w];
    const float* fro = nullptr;
    if (fk >= 0) {
        const float* ro = d.reach[o] + (size_t)(a == o ? it.rslot : it.oslot) * d.rstr[o];
        fro = ro;
        if (a == o) {  // the opponent folds with probability sigma_o[fk]
            float* rf = wsm + (size_t)w * d.nh_pad;
            for (int j = lane; j < nho; j += 32) {
                node_sigma<FMT, KA>(d, ar, it, loff, j, EVAL ? 1 : 0, sig);
                float sf = 0.0f;
#pragma unroll
                for (int k = 0; k < KA; k++)
                    if (k == fk) sf = sig[k];
                rf[j] = ro[j] * sf;
            }
            __syncwarp();
            fro = rf;
        }
        ftotal = warp_fold_sums(d, o, fro, s_S[w], fsc);
    }
    float* out = d.cfv + (size_t)it.cslot * d.nh_max;
    const float* cfv = d.cfv;
    const size_t stride = (size_t)d.nh_max;
#define CHILD_V(k, i) \
    ((k) == fk ? fold_value(d, p, (i), fro, ftotal, S, fsc, famount) : cfv[(size_t)cs[k] * stride + (i)])
    if (a != p) {  // opponent node: sum of children
        for (int i = lane; i < nh; i += 32) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) acc += CHILD_V(k, i);
            out[i] = acc;
        }
        return;
    }
    if (loff >= 0) {  // locked: fixed sigma, no update
        for (int i = lane; i < nh; i += 32) {
            float acc = 0.0f;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) acc += d.lock_sig[loff + (long long)k * nh + i] * CHILD_V(k, i);
            out[i] = acc;
        }
        return;
    }
    if (EVAL) {
        for (int i = lane; i < nh; i += 32) {
            float acc;
            if (mode == 0) {
                acc = CHILD_V(0, i);
#pragma unroll
                for (int k = 1; k < KA; k++)
                    if (k < na) {
                        const float v = CHILD_V(k, i);
                        if (v > acc) acc = v;
                    }
            } else {
                average_sigma<FMT, KA>(ar, a, it, i, sig);
                acc = 0.0f;
#pragma unroll
                for (int k = 0; k < KA; k++)
                    if (k < na) acc += sig[k] * CHILD_V(k, i);
            }
            out[i] = acc;
        }
        return;
    }
    const float pos = d.disc[0], neg = d.disc[1], ds = d.disc[2];
    const float* reach = d.reach[p] + (size_t)it.rslot * d.rstr[p];
    float v[KA];
    if (FMT == kDevF32) {
        float* R = (float*)ar.reg[p];
        float* Sg = (float*)ar.str[p];
        float* PR = (float*)ar.pred[p];
        for (int i = lane; i < nh; i += 32) {
            regret_sigma<FMT, KA>(ar, p, it, i, sig);
            float o_ = 0.0f;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    v[k] = CHILD_V(k, i);
                    o_ += sig[k] * v[k];
                }
            const float rp = reach[i];
            const size_t b = it.aoff + (size_t)i * na;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    const float r = R[b + k];
                    R[b + k] = r * (r > 0.0f ? pos : neg) + (v[k] - o_);
                    Sg[b + k] = Sg[b + k] * ds + rp * sig[k];
                    if (PR) PR[b + k] = v[k] - o_;
                }
            out[i] = o_;
        }
        return;
    }
    // 16-bit arenas (cfr.rs:350-407): pass 1 finds the node's new maxima
    // (warp reduction), pass 2 recomputes and requantises.
    int16_t* RQ = (int16_t*)ar.reg[p];
    uint16_t* SQ = (uint16_t*)ar.str[p];
    int16_t* PQ = (int16_t*)ar.pred[p];
    const float kr = ar.rscale[p][it.sidx] / 32767.0f;
    const float kss = ar.sscale[p][it.sidx] / 65535.0f * ds;
    const uint32_t sr_b = ar.sr ? sr_base(it.node, *d.iter) : 0u;
    float rmax = 0.0f, smax = 0.0f, pmax = 0.0f;
    for (int pass = 0; pass < 2; pass++) {
        float rk = 0.0f, sk = 0.0f, pk = 0.0f;
        if (pass == 1) {
            rmax = warp_max(rmax);
            smax = warp_max(smax);
            pmax = warp_max(pmax);
            rk = (rmax > 0.0f && isfinite(rmax)) ? 32767.0f / rmax : 0.0f;
            sk = (smax > 0.0f && isfinite(smax)) ? 65535.0f / smax : 0.0f;
            pk = (pmax > 0.0f && isfinite(pmax)) ? 32767.0f / pmax : 0.0f;
        }
        for (int i = lane; i < nh; i += 32) {
            regret_sigma<FMT, KA>(ar, p, it, i, sig);
            float o_ = 0.0f;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    v[k] = CHILD_V(k, i);
                    o_ += sig[k] * v[k];
                }
            const float rp = reach[i];
            const size_t b = it.aoff + (size_t)i * na;
#pragma unroll
            for (int k = 0; k < KA; k++)
                if (k < na) {
                    const int16_t qv = RQ[b + k];
                    const float nr = (float)qv * kr * (qv > 0 ? pos : neg) + (v[k] - o_);
                    const float ns = (float)SQ[b + k] * kss + rp * sig[k];
                    if (pass == 0) {
                        rmax = fmaxf(rmax, fabsf(nr));
                        smax = fmaxf(smax, ns);
                        if (PQ) pmax = fmaxf(pmax, fabsf(v[k] - o_));
                    } else {
                        requant16(nr, ns, rk, sk, ar.sr, sr_b, i, k, &RQ[b + k], &SQ[b + k]);
                        if (PQ) PQ[b + k] = pk > 0.0f ? sat_i16((v[k] - o_) * pk) : (int16_t)0;
                    }
                }
            if (pass == 1) out[i] = o_;
        }
        __syncwarp();  // every lane has read the old quants of its hands before any scale changes
    }
#undef CHILD_V
    if (lane == 0) {
        ar.rscale[p][it.sidx] = (rmax > 0.0f && isfinite(rmax)) ? rmax : 0.0f;
        ar.sscale[p][it.sidx] = (smax > 0.0f && isfinite(smax)) ? smax : 0.0f;
        if (PQ) ar.pscale[p][it.sidx] = (pmax > 0.0f && isfinite(pmax)) ? pmax : 0.0f;
    }
}

// sum_i w_p[i] * cfv_root[i] in f64 (best_response.rs:263-269).
__global__ void __launch_bounds__(kThreads) k_root_dot(Dev d, int p, int slot) {
    __shared__ double s_red[kWarps];
    double v = 0.0;
    for (int i = threadIdx.x; i < d.nh[p]; i += blockDim.x) v += (double)d.w[p][i] * (double)d.cfv[i];
    v = block_sum<double>(v, s_red);
    if (threadIdx.x == 0) d.dot[slot] = v;
}

// Arena import / export between the reference layout (action-major f32 or
// quants at data_offset) and the device layout (hand-major, 16-aligned).
struct XNode { uint64_t host_off, dev_off; uint32_t na, sidx; };
template <class T>
__global__ void k_to_host(const T* dev, T* host, const XNode* xs, int nh) {
    const XNode x = xs[blockIdx.x];
    for (int i = threadIdx.x; i < nh; i += blockDim.x)
        for (uint32_t k = 0; k < x.na; k++) host[x.host_off + (size_t)k * nh + i] = dev[x.dev_off + (size_t)i * x.na + k];
}
template <class T>
__global__ void k_to_dev(const T* host, T* dev, const XNode* xs, int nh) {
    const XNode x = xs[blockIdx.x];
    for (int i = threadIdx.x; i < nh; i += blockDim.x)
        for (uint32_t k = 0; k < x.na; k++) dev[x.dev_off + (size_t)i * x.na + k] = host[x.host_off + (size_t)k * nh + i];
}
template <class T>
__global__ void k_decode_to_host(const T* dev, const float* scale, float* host, const XNode* xs, int nh, float div) {
    const XNode x = xs[blockIdx.x];
    const float kq = scale[x.sidx] / div;
    for (int i = threadIdx.x; i < nh; i += blockDim.x)
        for (uint32_t k = 0; k < x.na; k++)
            host[x.host_off + (size_t)k * nh + i] = (float)dev[x.dev_off + (size_t)i * x.na + k] * kq;
}
// encode f32 host blocks into 16-bit device blocks (store.rs:199-215)
__global__ void __launch_bounds__(kThreads) k_encode(const float* host, void* dev, float* scale, const XNode* xs, int nh,
                                                     int is_unsigned) {
    __shared__ float s_max[kWarps];
    const XNode x = xs[blockIdx.x];
    const size_t n = (size_t)x.na * nh;
    float m = 0.0f;
    for (size_t t = threadIdx.x; t < n; t += blockDim.x) {
        const float v = host[x.host_off + t];
        m = is_unsigned ? fmaxf(m, v) : fmaxf(m, fabsf(v));
    }
    m = block_max(m, s_max);
    const bool ok = m > 0.0f && isfinite(m);
    const float kq = ok ? (is_unsigned ? 65535.0f : 32767.0f) / m : 0.0f;
    for (size_t t = threadIdx.x; t < n; t += blockDim.x) {
        const size_t k = t / nh, i = t % nh;
        const float v = host[x.host_off + t];
        const size_t di = x.dev_off + i * x.na + k;
        if (is_unsigned) ((uint16_t*)dev)[di] = ok ? sat_u16(fmaxf(v, 0.0f) * kq) : (uint16_t)0;
        else ((int16_t*)dev)[di] = ok ? sat_i16(v * kq) : (int16_t)0;
    }
    if (threadIdx.x == 0) scale[x.sidx] = ok ? m : 0.0f;
}
// The FP8 twins of k_encode / k_decode_to_host: v * (448 / max) per node and
// back, max kept as the node's scale (strategy sums clamped at 0).
__global__ void __launch_bounds__(kThreads) k_encode_fp8(const float* host, uint8_t* dev, float* scale, const XNode* xs,
                                                         int nh, int is_unsigned) {
    __shared__ float s_max[kWarps];
    const XNode x = xs[blockIdx.x];
    const size_t n = (size_t)x.na * nh;
    float m = 0.0f;
    for (size_t t = threadIdx.x; t < n; t += blockDim.x) {
        const float v = host[x.host_off + t];
        m = is_unsigned ? fmaxf(m, v) : fmaxf(m, fabsf(v));
    }
    m = block_max(m, s_max);
    const bool ok = m > 0.0f && isfinite(m);
    const float kq = ok ? 448.0f / m : 0.0f;
    for (size_t t = threadIdx.x; t < n; t += blockDim.x) {
        const size_t k = t / nh, i = t % nh;
        const float v = host[x.host_off + t];
        dev[x.dev_off + i * x.na + k] = ok ? f32_to_e4m3(is_unsigned ? fmaxf(v, 0.0f) * kq : v * kq) : (uint8_t)0;
    }
    if (threadIdx.x == 0) scale[x.sidx] = ok ? m : 0.0f;
}
__global__ void k_decode_fp8_to_host(const uint8_t* dev, const float* scale, float* host, const XNode* xs, int nh) {
    const XNode x = xs[blockIdx.x];
    const float kq = scale[x.sidx] / 448.0f;
    for (int i = threadIdx.x; i < nh; i += blockDim.x)
        for (uint32_t k = 0; k < x.na; k++)
            host[x.host_off + (size_t)k * nh + i] = e4m3_to_f32(dev[x.dev_off + (size_t)i * x.na + k]) * kq;
}

}  // namespace gtob
