// Level-synchronous discounted-CFR engine for sm_100a.
//
// One iteration = for traverser p in {0, 1}: a down sweep writing reach
// vectors level by level, then an up sweep evaluating terminals and folding
// counterfactual values (with the DCFR / CFR+ / PCFR+ regret and strategy-sum
// update) back to the root -- the work split of the reference's
// gpu/kernels.cu and gpu/mod.rs:622-841, re-designed:
//   * work items carry precomputed slot indices (plan.hpp); reach and cfv
//     vectors live in compact slots;
//   * arenas are hand-major per node, f32 or 16-bit with a per-node scale
//     (requantised in-kernel after a block max), matching cfr.rs:297-409;
//   * terminal sums are deterministic f64 reductions (fold: per-card sums;
//     showdown: strength-sorted prefix scans with per-card corrections and
//     precomputed ranks) mirroring game.rs:470-577;
//   * discounts are computed on the device in f64 from a device iteration
//     counter, so one captured CUDA graph replays every iteration.
// The file is compiled with -fmad=false: every multiply and add rounds
// separately, as the reference's f32 arithmetic does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "engine.hpp"

namespace gtob {

const char* const kKernelNames[7] = {"copy_root", "down_action", "down_chance", "up_fold",
                                     "up_show",   "up_chance",   "up_action"};

#define CK(x)                                                                                     \
    do {                                                                                          \
        cudaError_t e_ = (x);                                                                     \
        if (e_ != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(e_) + " at " #x); \
    } while (0)

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// ------------------------------------------------------------ device state
struct Dev {
    int nh[2];
    int nh_max;
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
    const uint32_t* rank_off[2];
    const uint32_t* rank_cnt[2];
    const RankEntry* rank[2];
    const CardEntry* cards;
    float* reach[2];
    float* cfv;
    const long long* lock_off[2];  // per sidx, -1 = unlocked
    const float* lock_sig;
    float* disc;  // pos, neg, strat
    unsigned* iter;
    double* dot;  // root dot products
};
struct Arenas {
    void* reg[2];
    void* str[2];
    void* pred[2];  // PCFR+ only, else null
    float* rscale[2];
    float* sscale[2];
    float* pscale[2];
};

// ----------------------------------------------------------- small helpers
__device__ __forceinline__ int16_t sat_i16(float x) {  // Rust `as i16` after round-ties-even
    if (x != x) return 0;
    float r = rintf(x);
    r = fminf(fmaxf(r, -32768.0f), 32767.0f);
    return (int16_t)r;
}
__device__ __forceinline__ uint16_t sat_u16(float x) {
    if (x != x) return 0;
    float r = rintf(x);
    r = fminf(fmaxf(r, 0.0f), 65535.0f);
    return (uint16_t)r;
}
__device__ __forceinline__ float block_max(float v, float* sh) {
    // order-independent (max), so deterministic
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    float m = sh[0];
    for (int k = 1; k < kWarps; k++) m = fmaxf(m, sh[k]);
    return m;
}
__device__ __forceinline__ double block_sum_f64(double v, double* sh) {
    // fixed tree: deterministic for a fixed launch shape
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
    for (int k = 0; k < kWarps; k++) s += sh[k];
    return s;
}

// Current strategy of one hand at an action node (cfr.rs:240-292, 875-942).
// Writes sig[0..na); entries of hand i are arena[aoff + i*na + k].
template <int FMT>
__device__ __forceinline__ void regret_sigma(const Arenas& ar, int actor, const ActItem& it, int i, float* sig) {
    const int na = (int)it.na;
    const size_t base = it.aoff + (size_t)i * na;
    if (FMT == kFmtF32) {
        const float* r = (const float*)ar.reg[actor] + base;
        if (ar.pred[actor]) {
            const float* pr = (const float*)ar.pred[actor] + base;
            float sum = 0.0f;
            for (int k = 0; k < na; k++) {
                sig[k] = fmaxf(r[k], 0.0f) + pr[k];
                sum += fmaxf(sig[k], 0.0f);
            }
            if (sum > 1e-12f) {
                const float inv = 1.0f / sum;
                for (int k = 0; k < na; k++) sig[k] = fmaxf(sig[k], 0.0f) * inv;
            } else {
                const float u = 1.0f / (float)na;
                for (int k = 0; k < na; k++) sig[k] = u;
            }
        } else {
            float sum = 0.0f;
            for (int k = 0; k < na; k++) sum += fmaxf(r[k], 0.0f);
            if (sum > 1e-12f) {
                const float inv = 1.0f / sum;
                for (int k = 0; k < na; k++) sig[k] = fmaxf(r[k], 0.0f) * inv;
            } else {
                const float u = 1.0f / (float)na;
                for (int k = 0; k < na; k++) sig[k] = u;
            }
        }
    } else {
        const int16_t* q = (const int16_t*)ar.reg[actor] + base;
        if (ar.pred[actor]) {
            const int16_t* qp = (const int16_t*)ar.pred[actor] + base;
            const float kr = ar.rscale[actor][it.sidx] / 32767.0f;
            const float kp = ar.pscale[actor][it.sidx] / 32767.0f;
            float sum = 0.0f;
            for (int k = 0; k < na; k++) {
                sig[k] = (float)max((int)q[k], 0) * kr + (float)qp[k] * kp;
                sum += fmaxf(sig[k], 0.0f);
            }
            if (sum > 1e-12f) {
                const float inv = 1.0f / sum;
                for (int k = 0; k < na; k++) sig[k] = fmaxf(sig[k], 0.0f) * inv;
            } else {
                const float u = 1.0f / (float)na;
                for (int k = 0; k < na; k++) sig[k] = u;
            }
        } else {
            int sum = 0;
            for (int k = 0; k < na; k++) sum += max((int)q[k], 0);
            if (sum > 0) {
                const float inv = 1.0f / (float)sum;
                for (int k = 0; k < na; k++) sig[k] = (float)max((int)q[k], 0) * inv;
            } else {
                const float u = 1.0f / (float)na;
                for (int k = 0; k < na; k++) sig[k] = u;
            }
        }
    }
}
// Average strategy of one hand (cfr.rs:679-726).
template <int FMT>
__device__ __forceinline__ void average_sigma(const Arenas& ar, int actor, const ActItem& it, int i, float* sig) {
    const int na = (int)it.na;
    const size_t base = it.aoff + (size_t)i * na;
    if (FMT == kFmtF32) {
        const float* s = (const float*)ar.str[actor] + base;
        double sum = 0.0;
        for (int k = 0; k < na; k++) sum += (double)fmaxf(s[k], 0.0f);
        if (sum > 1e-12) {
            for (int k = 0; k < na; k++) sig[k] = (float)((double)fmaxf(s[k], 0.0f) / sum);
        } else {
            const float u = 1.0f / (float)na;
            for (int k = 0; k < na; k++) sig[k] = u;
        }
    } else {
        const uint16_t* q = (const uint16_t*)ar.str[actor] + base;
        unsigned sum = 0;
        for (int k = 0; k < na; k++) sum += q[k];
        if (sum > 0) {
            const float inv = 1.0f / (float)sum;
            for (int k = 0; k < na; k++) sig[k] = (float)q[k] * inv;
        } else {
            const float u = 1.0f / (float)na;
            for (int k = 0; k < na; k++) sig[k] = u;
        }
    }
}

constexpr int kMaxActions = 32;  // register cache bound; nodes above it are rejected at plan time

// ------------------------------------------------------------------ kernels
__global__ void k_begin_iteration(unsigned* iter, float* disc, int algo) {
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

__global__ void k_copy_root(Dev d) {
    for (int q = 0; q < 2; q++)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.nh[q]; i += gridDim.x * blockDim.x)
            d.reach[q][i] = d.w[q][i];
}

// Down sweep, action nodes: child actor reach = parent reach * sigma.
// mode 0: current strategy (regret matching), mode 1: average strategy.
template <int FMT>
__global__ void __launch_bounds__(kThreads) k_down_action(Dev d, Arenas ar, const ActItem* items, int mode) {
    const ActItem it = items[blockIdx.x];
    const int a = (int)it.actor, na = (int)it.na, nh = d.nh[a];
    const float* parent = d.reach[a] + (size_t)it.rslot * nh;
    float* child = d.reach[a] + (size_t)it.child_rslot * nh;
    const long long loff = d.lock_off[a][it.sidx];
    float sig[kMaxActions];
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
        const float pr = parent[i];
        if (loff >= 0) {
            for (int k = 0; k < na; k++) sig[k] = d.lock_sig[loff + (long long)k * nh + i];
        } else if (mode == 0) {
            regret_sigma<FMT>(ar, a, it, i, sig);
        } else {
            average_sigma<FMT>(ar, a, it, i, sig);
        }
        for (int k = 0; k < na; k++) child[(size_t)k * nh + i] = pr * sig[k];
    }
}

// Down sweep, chance edges: both players' reach with holders of the card zeroed.
__global__ void __launch_bounds__(kThreads) k_down_chance(Dev d, const EdgeItem* items) {
    const EdgeItem e = items[blockIdx.x];
    for (int q = 0; q < 2; q++) {
        const int nh = d.nh[q];
        const float* pr = d.reach[q] + (size_t)e.prs[q] * nh;
        float* cr = d.reach[q] + (size_t)e.crs[q] * nh;
        for (int i = threadIdx.x; i < nh; i += blockDim.x) cr[i] = (d.mask[q][i] >> e.card & 1ull) ? 0.0f : pr[i];
    }
}

// Fold terminal (game.rs:470-496): amount * (compatible opponent reach), with
// the total and per-card sums as deterministic f64 reductions.
__global__ void __launch_bounds__(kThreads) k_fold(Dev d, const FoldItem* items, int p) {
    __shared__ double s_card[52];
    __shared__ double s_red[kWarps];
    const FoldItem f = items[blockIdx.x];
    const int o = 1 - p, nho = d.nh[o], nhp = d.nh[p];
    const float* ro = d.reach[o] + (size_t)f.rs[o] * nho;
    double t = 0.0;
    for (int j = threadIdx.x; j < nho; j += blockDim.x) t += (double)ro[j];
    const double total = block_sum_f64(t, s_red);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = warp; c < 52; c += kWarps) {
        const uint32_t b = d.hcard_off[o][c], e = d.hcard_off[o][c + 1];
        double v = 0.0;
        for (uint32_t k = b + lane; k < e; k += 32) v += (double)ro[d.hcard_idx[o][k]];
        for (int x = 16; x > 0; x >>= 1) v += __shfl_xor_sync(0xffffffffu, v, x);
        if (lane == 0) s_card[c] = v;
    }
    __syncthreads();
    const float amount = (int)f.folder == p ? f.tlose : f.twin;
    float* out = d.cfv + (size_t)f.cslot * d.nh_max;
    for (int i = threadIdx.x; i < nhp; i += blockDim.x) {
        const uint32_t sm = d.same[p][i];
        const float same_r = sm != kSentinel ? ro[sm] : 0.0f;
        const float valid = (float)(total - s_card[d.c1[p][i]] - s_card[d.c2[p][i]]) + same_r;
        out[i] = amount * valid;
    }
}

// Block exclusive scan of x[0..m) into out[0..m], out[m] = total (f64, fixed order).
__device__ void block_exclusive_scan(const double* x, double* out, int m, double* s_w) {
    const int tid = threadIdx.x;
    const int chunk = (m + kThreads - 1) / kThreads;
    const int lo = min(tid * chunk, m), hi = min(lo + chunk, m);
    double local = 0.0;
    for (int k = lo; k < hi; k++) local += x[k];
    double incl = local;
    const int lane = tid & 31, warp = tid >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        double y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    double wbase = 0.0;
    for (int k = 0; k < warp; k++) wbase += s_w[k];
    double run = wbase + (incl - local);
    for (int k = lo; k < hi; k++) {
        out[k] = run;
        run += x[k];
    }
    if (tid == kThreads - 1) {
        double tot = 0.0;
        for (int k = 0; k < kWarps; k++) tot += s_w[k];
        out[m] = tot;
    }
    __syncthreads();
}

// Showdown terminal (game.rs:501-577) as a strength-sorted prefix scan with
// card-removal corrections.  Shared memory: R (sorted opp reach), P (its
// exclusive prefix, P[m] = total), Q (per-card exclusive prefixes).
__global__ void __launch_bounds__(kThreads) k_showdown(Dev d, const ShowItem* items, int p) {
    extern __shared__ double sh[];
    __shared__ double s_w[kWarps];
    const ShowItem s = items[blockIdx.x];
    const int o = 1 - p, nho = d.nh[o], nhp = d.nh[p];
    const int m = (int)d.sorted_cnt[o][s.slot];
    const uint16_t* sidx = d.sorted_idx[o] + d.sorted_off[o][s.slot];
    const uint32_t* coff = d.ccard_off[o] + (size_t)s.slot * 53;
    const uint16_t* cpos = d.ccard_pos[o];
    const float* ro = d.reach[o] + (size_t)s.rs[o] * nho;
    double* R = sh;
    double* P = R + m;
    double* Q = P + m + 1;
    for (int k = threadIdx.x; k < m; k += blockDim.x) R[k] = (double)ro[sidx[k]];
    float* out = d.cfv + (size_t)s.cslot * d.nh_max;
    for (int i = threadIdx.x; i < nhp; i += blockDim.x) out[i] = 0.0f;
    __syncthreads();
    block_exclusive_scan(R, P, m, s_w);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t c0 = coff[0];
    for (int c = warp; c < 52; c += kWarps) {
        const uint32_t b = coff[c], e = coff[c + 1];
        double* q = Q + (b - c0) + c;
        double carry = 0.0;
        if (lane == 0) q[0] = 0.0;
        for (uint32_t k0 = b; k0 < e; k0 += 32) {
            const uint32_t k = k0 + lane;
            double v = k < e ? R[cpos[k]] : 0.0;
            for (int x = 1; x < 32; x <<= 1) {
                double y = __shfl_up_sync(0xffffffffu, v, x);
                if (lane >= x) v += y;
            }
            if (k < e) q[k - b + 1] = carry + v;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
    }
    __syncthreads();
    const double total = P[m];
    const int mp = (int)d.rank_cnt[p][s.slot];
    const RankEntry* re = d.rank[p] + d.rank_off[p][s.slot];
    for (int k = threadIdx.x; k < mp; k += blockDim.x) {
        const RankEntry e = re[k];
        const int h = e.idx;
        const int a1 = d.c1[p][h], a2 = d.c2[p][h];
        const double* q1 = Q + (coff[a1] - c0) + a1;
        const double* q2 = Q + (coff[a2] - c0) + a2;
        const double t1 = q1[coff[a1 + 1] - coff[a1]], t2 = q2[coff[a2 + 1] - coff[a2]];
        const float lower = (float)(P[e.lb] - q1[e.c1lo] - q2[e.c2lo]);
        const float higher = (float)((total - P[e.ub]) - (t1 - q1[e.c1hi]) - (t2 - q2[e.c2hi]));
        const uint32_t sm = d.same[p][h];
        const float same_r = sm != kSentinel ? ro[sm] : 0.0f;
        const float valid = (float)(total - t1 - t2) + same_r;
        const float tied = valid - lower - higher;
        out[h] = s.twin * lower + s.tlose * higher + s.ttie * tied;
    }
}

// Chance node (cfr.rs:637-663): sum of representative children through the
// suit-permutation hand tables, skipping holders of the card, times 1/divisor.
__global__ void __launch_bounds__(kThreads) k_chance(Dev d, const ChanceItem* items, int p) {
    const ChanceItem c = items[blockIdx.x];
    const int nh = d.nh[p];
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
        const uint64_t hm = d.mask[p][i];
        float acc = 0.0f;
        for (uint32_t t = c.cc_start; t < c.cc_start + c.cc_count; t++) {
            const CardEntry e = d.cards[t];
            if (hm >> e.card & 1ull) continue;
            const int src = e.perm ? (int)d.hperm[p][(size_t)e.perm * nh + i] : i;
            acc += d.cfv[(size_t)e.child_cslot * d.nh_max + src];
        }
        d.cfv[(size_t)c.cslot * d.nh_max + i] = acc * c.inv;
    }
}

// Up sweep, action nodes, CFR update (cfr.rs:469-531 with update_node 297-409).
template <int FMT>
__global__ void __launch_bounds__(kThreads) k_up_action(Dev d, Arenas ar, const ActItem* items, int p) {
    __shared__ float s_max[kWarps];
    const ActItem it = items[blockIdx.x];
    const int a = (int)it.actor, na = (int)it.na, nh = d.nh[p];
    float* out = d.cfv + (size_t)it.cslot * d.nh_max;
    const float* cv = d.cfv + (size_t)it.child_cslot * d.nh_max;
    const size_t stride = (size_t)d.nh_max;
    if (a != p) {  // opponent node: sum of children
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            float acc = 0.0f;
            for (int k = 0; k < na; k++) acc += cv[k * stride + i];
            out[i] = acc;
        }
        return;
    }
    const long long loff = d.lock_off[a][it.sidx];
    if (loff >= 0) {  // locked: fixed sigma, no update
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            float acc = 0.0f;
            for (int k = 0; k < na; k++) acc += d.lock_sig[loff + (long long)k * nh + i] * cv[k * stride + i];
            out[i] = acc;
        }
        return;
    }
    const float pos = d.disc[0], neg = d.disc[1], ds = d.disc[2];
    const float* reach = d.reach[p] + (size_t)it.rslot * nh;
    float sig[kMaxActions];
    if (FMT == kFmtF32) {
        float* R = (float*)ar.reg[p];
        float* S = (float*)ar.str[p];
        float* PR = (float*)ar.pred[p];
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            regret_sigma<FMT>(ar, p, it, i, sig);
            float o = 0.0f;
            for (int k = 0; k < na; k++) o += sig[k] * cv[k * stride + i];
            const float rp = reach[i];
            const size_t b = it.aoff + (size_t)i * na;
            for (int k = 0; k < na; k++) {
                const float v = cv[k * stride + i];
                const float r = R[b + k];
                R[b + k] = r * (r > 0.0f ? pos : neg) + (v - o);
                S[b + k] = S[b + k] * ds + rp * sig[k];
                if (PR) PR[b + k] = v - o;
            }
            out[i] = o;
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
    float rmax = 0.0f, smax = 0.0f, pmax = 0.0f;
    for (int pass = 0; pass < 2; pass++) {
        float rk = 0.0f, sk = 0.0f, pk = 0.0f;
        if (pass == 1) {
            rmax = block_max(rmax, s_max);
            smax = block_max(smax, s_max);
            if (PQ) pmax = block_max(pmax, s_max);
            rk = (rmax > 0.0f && isfinite(rmax)) ? 32767.0f / rmax : 0.0f;
            sk = (smax > 0.0f && isfinite(smax)) ? 65535.0f / smax : 0.0f;
            pk = (pmax > 0.0f && isfinite(pmax)) ? 32767.0f / pmax : 0.0f;
        }
        for (int i = threadIdx.x; i < nh; i += blockDim.x) {
            regret_sigma<FMT>(ar, p, it, i, sig);
            float o = 0.0f;
            for (int k = 0; k < na; k++) o += sig[k] * cv[k * stride + i];
            const float rp = reach[i];
            const size_t b = it.aoff + (size_t)i * na;
            float nr[kMaxActions], ns[kMaxActions];
            for (int k = 0; k < na; k++) {
                const float v = cv[k * stride + i];
                const int16_t qv = RQ[b + k];
                nr[k] = (float)qv * kr * (qv > 0 ? pos : neg) + (v - o);
                ns[k] = (float)SQ[b + k] * kss + rp * sig[k];
            }
            if (pass == 0) {
                for (int k = 0; k < na; k++) {
                    rmax = fmaxf(rmax, fabsf(nr[k]));
                    smax = fmaxf(smax, ns[k]);
                    if (PQ) pmax = fmaxf(pmax, fabsf(cv[k * stride + i] - o));
                }
            } else {
                for (int k = 0; k < na; k++) {
                    const float v = cv[k * stride + i];
                    RQ[b + k] = rk > 0.0f ? sat_i16(nr[k] * rk) : (int16_t)0;
                    SQ[b + k] = sk > 0.0f ? sat_u16(fmaxf(ns[k], 0.0f) * sk) : (uint16_t)0;
                    if (PQ) PQ[b + k] = pk > 0.0f ? sat_i16((v - o) * pk) : (int16_t)0;
                }
                out[i] = o;
            }
        }
    }
    __syncthreads();  // every thread has read the old scales
    if (threadIdx.x == 0) {
        ar.rscale[p][it.sidx] = (rmax > 0.0f && isfinite(rmax)) ? rmax : 0.0f;
        ar.sscale[p][it.sidx] = (smax > 0.0f && isfinite(smax)) ? smax : 0.0f;
        if (PQ) ar.pscale[p][it.sidx] = (pmax > 0.0f && isfinite(pmax)) ? pmax : 0.0f;
    }
}

// Up sweep, action nodes, evaluation (best_response.rs:69-121, 185-219):
// mode 0 best response (max over actions), mode 1 average strategy.
template <int FMT>
__global__ void __launch_bounds__(kThreads) k_up_eval(Dev d, Arenas ar, const ActItem* items, int p, int mode) {
    const ActItem it = items[blockIdx.x];
    const int a = (int)it.actor, na = (int)it.na, nh = d.nh[p];
    float* out = d.cfv + (size_t)it.cslot * d.nh_max;
    const float* cv = d.cfv + (size_t)it.child_cslot * d.nh_max;
    const size_t stride = (size_t)d.nh_max;
    const long long loff = a == p ? d.lock_off[a][it.sidx] : -1;
    float sig[kMaxActions];
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
        float acc = 0.0f;
        if (a != p) {
            for (int k = 0; k < na; k++) acc += cv[k * stride + i];
        } else if (loff >= 0) {
            for (int k = 0; k < na; k++) acc += d.lock_sig[loff + (long long)k * nh + i] * cv[k * stride + i];
        } else if (mode == 0) {
            acc = cv[i];
            for (int k = 1; k < na; k++) {
                const float v = cv[k * stride + i];
                if (v > acc) acc = v;
            }
        } else {
            average_sigma<FMT>(ar, a, it, i, sig);
            for (int k = 0; k < na; k++) acc += sig[k] * cv[k * stride + i];
        }
        out[i] = acc;
    }
}

// sum_i w_p[i] * cfv_root[i] in f64 (best_response.rs:263-269).
__global__ void __launch_bounds__(kThreads) k_root_dot(Dev d, int p, int slot) {
    __shared__ double s_red[kWarps];
    double v = 0.0;
    for (int i = threadIdx.x; i < d.nh[p]; i += blockDim.x) v += (double)d.w[p][i] * (double)d.cfv[i];
    v = block_sum_f64(v, s_red);
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
// decode 16-bit device blocks to f32 host layout
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

// ------------------------------------------------------------- host engine
template <class T>
static T* dupload(const std::vector<T>& v, std::vector<void*>& owned, size_t* bytes) {
    T* p = nullptr;
    const size_t n = std::max<size_t>(v.size(), 1);
    CK(cudaMalloc(&p, n * sizeof(T)));
    owned.push_back(p);
    *bytes += n * sizeof(T);
    if (!v.empty()) CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return p;
}
static void* dalloc(size_t bytes, std::vector<void*>& owned, size_t* total) {
    void* p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
    owned.push_back(p);
    *total += bytes;
    CK(cudaMemset(p, 0, std::max<size_t>(bytes, 16)));
    return p;
}

struct EngineImpl {
    const Spot* spot;
    Plan plan;
    int fmt = kFmtF32;
    int algo = kDcfr;
    bool pcfr = false;
    uint32_t iteration = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> owned;
    size_t bytes = 0;
    Dev d{};
    Arenas ar{};
    // device copies of work lists
    ActItem* act = nullptr;
    EdgeItem* edge = nullptr;
    FoldItem* fold = nullptr;
    ShowItem* show = nullptr;
    ChanceItem* chance = nullptr;
    XNode* xnodes[2] = {nullptr, nullptr};
    std::vector<XNode> hx[2];
    void* lock_buf = nullptr;
    long long* lock_off_dev[2] = {nullptr, nullptr};
    float* staging = nullptr;  // device f32 image of one arena in the reference layout
    float* pinned = nullptr;
    size_t staging_len = 0;
    size_t show_smem = 0;
    cudaGraphExec_t g_iter = nullptr;
    cudaGraphExec_t g_eval[2] = {nullptr, nullptr};
    double* h_dot = nullptr;  // pinned

    ~EngineImpl() {
        if (stream) cudaStreamSynchronize(stream);
        if (g_iter) cudaGraphExecDestroy(g_iter);
        for (auto& g : g_eval)
            if (g) cudaGraphExecDestroy(g);
        if (lock_buf) cudaFree(lock_buf);
        for (void* p : owned) cudaFree(p);
        if (pinned) cudaFreeHost(pinned);
        if (h_dot) cudaFreeHost(h_dot);
        if (stream) cudaStreamDestroy(stream);
    }

    void upload_locks(const HostSolver& host) {
        if (lock_buf) {
            CK(cudaStreamSynchronize(stream));
            CK(cudaFree(lock_buf));
            lock_buf = nullptr;
        }
        std::vector<long long> off[2];
        std::vector<float> sig;
        for (int p = 0; p < 2; p++) off[p].assign(std::max<uint64_t>(plan.n_anodes[p], 1), -1);
        for (auto& kv : host.locks) {
            const int32_t s = plan.node_sidx[kv.first];
            if (s < 0) continue;  // lock on a branch the device does not traverse
            off[spot->tree.player[kv.first]][s] = (long long)sig.size();
            sig.insert(sig.end(), kv.second.begin(), kv.second.end());
        }
        if (sig.empty()) sig.push_back(0.0f);
        const size_t b0 = off[0].size() * 8, b1 = off[1].size() * 8, bs = sig.size() * 4;
        CK(cudaMalloc(&lock_buf, b0 + b1 + bs));
        char* base = (char*)lock_buf;
        CK(cudaMemcpy(base, off[0].data(), b0, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(base + b0, off[1].data(), b1, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(base + b0 + b1, sig.data(), bs, cudaMemcpyHostToDevice));
        d.lock_off[0] = (const long long*)base;
        d.lock_off[1] = (const long long*)(base + b0);
        d.lock_sig = (const float*)(base + b0 + b1);
        drop_graphs();
    }
    void drop_graphs() {
        if (g_iter) { cudaGraphExecDestroy(g_iter); g_iter = nullptr; }
        for (auto& g : g_eval)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    template <class F>
    void timed(Profile* pr, int kind, F launch) {
        if (!pr) { launch(); return; }
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        CK(cudaEventRecord(a, stream));
        launch();
        CK(cudaEventRecord(b, stream));
        CK(cudaEventSynchronize(b));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, a, b));
        pr->ms[kind] += ms;
        pr->launches[kind] += 1;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }

    // One sweep for traverser p.  eval < 0: CFR iteration; 0/1: BR / average.
    void sweep(int p, int eval, Profile* pr) {
        timed(pr, 0, [&] { k_copy_root<<<4, kThreads, 0, stream>>>(d); });
        const int L = plan.num_levels;
        const int down_mode = eval < 0 ? 0 : 1;
        for (int l = 0; l < L; l++) {
            const Span sa = plan.act_span[l];
            if (sa.count)
                timed(pr, 1, [&] {
                    if (fmt == kFmtF32) k_down_action<kFmtF32><<<sa.count, kThreads, 0, stream>>>(d, ar, act + sa.start, down_mode);
                    else k_down_action<kFmtI16><<<sa.count, kThreads, 0, stream>>>(d, ar, act + sa.start, down_mode);
                });
            const Span se = plan.edge_span[l];
            if (se.count) timed(pr, 2, [&] { k_down_chance<<<se.count, kThreads, 0, stream>>>(d, edge + se.start); });
        }
        for (int l = L - 1; l >= 0; l--) {
            const Span sf = plan.fold_span[l];
            if (sf.count) timed(pr, 3, [&] { k_fold<<<sf.count, kThreads, 0, stream>>>(d, fold + sf.start, p); });
            const Span ss = plan.show_span[l];
            if (ss.count)
                timed(pr, 4, [&] { k_showdown<<<ss.count, kThreads, show_smem, stream>>>(d, show + ss.start, p); });
            const Span sc = plan.chance_span[l];
            if (sc.count) timed(pr, 5, [&] { k_chance<<<sc.count, kThreads, 0, stream>>>(d, chance + sc.start, p); });
            const Span sa = plan.act_span[l];
            if (sa.count)
                timed(pr, 6, [&] {
                    if (eval < 0) {
                        if (fmt == kFmtF32) k_up_action<kFmtF32><<<sa.count, kThreads, 0, stream>>>(d, ar, act + sa.start, p);
                        else k_up_action<kFmtI16><<<sa.count, kThreads, 0, stream>>>(d, ar, act + sa.start, p);
                    } else {
                        if (fmt == kFmtF32) k_up_eval<kFmtF32><<<sa.count, kThreads, 0, stream>>>(d, ar, act + sa.start, p, eval);
                        else k_up_eval<kFmtI16><<<sa.count, kThreads, 0, stream>>>(d, ar, act + sa.start, p, eval);
                    }
                });
        }
        CK(cudaGetLastError());
    }
    void record_iteration() {
        k_begin_iteration<<<1, 1, 0, stream>>>(d.iter, d.disc, algo);
        sweep(0, -1, nullptr);
        sweep(1, -1, nullptr);
    }
    void record_eval(int mode) {
        for (int p = 0; p < 2; p++) {
            sweep(p, mode, nullptr);
            k_root_dot<<<1, kThreads, 0, stream>>>(d, p, p);
        }
        CK(cudaMemcpyAsync(h_dot, d.dot, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    }
    cudaGraphExec_t capture(int which) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            if (which < 0) record_iteration();
            else record_eval(which);
        } catch (...) {
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        CK(cudaStreamEndCapture(stream, &g));
        cudaGraphExec_t ex;
        CK(cudaGraphInstantiate(&ex, g, 0));
        cudaGraphDestroy(g);
        return ex;
    }
};

// --------------------------------------------------------------- GpuEngine
GpuEngine::GpuEngine(const HostSolver& host, int fmt) : d_(new EngineImpl()) {
    EngineImpl& E = *d_;
    const Spot& sp = *host.spot;
    E.spot = &sp;
    E.algo = host.algo;
    E.pcfr = host.algo == kPcfrPlus;
    E.fmt = fmt < 0 ? (host.storage == kStoreF32 ? kFmtF32 : kFmtI16) : fmt;
    if (E.fmt != kFmtF32 && E.fmt != kFmtI16) throw Error("unknown device arena format");
    E.iteration = host.iteration;
    E.plan = build_plan(sp, host.use_iso);
    const Plan& P = E.plan;
    for (auto& a : P.act)
        if ((int)a.na > kMaxActions) throw Error("action node with more than 32 actions is not supported on the GPU");
    CK(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
    size_t& B = E.bytes;
    auto& O = E.owned;
    Dev& d = E.d;
    d.nh[0] = P.nh[0];
    d.nh[1] = P.nh[1];
    d.nh_max = P.nh_max;
    for (int q = 0; q < 2; q++) {
        const Hands& h = sp.hands[q];
        d.c1[q] = dupload(h.c1, O, &B);
        d.c2[q] = dupload(h.c2, O, &B);
        d.mask[q] = dupload(h.mask, O, &B);
        d.same[q] = dupload(sp.same[q], O, &B);
        d.w[q] = dupload(h.w, O, &B);
        std::vector<uint16_t> hp;
        for (auto& t : sp.hand_perm[q]) hp.insert(hp.end(), t.begin(), t.end());
        d.hperm[q] = dupload(hp, O, &B);
        d.hcard_off[q] = dupload(P.hcard_off[q], O, &B);
        d.hcard_idx[q] = dupload(P.hcard_idx[q], O, &B);
        d.sorted_off[q] = dupload(P.sorted_off[q], O, &B);
        d.sorted_cnt[q] = dupload(P.sorted_cnt[q], O, &B);
        d.sorted_idx[q] = dupload(P.sorted_idx[q], O, &B);
        d.ccard_off[q] = dupload(P.ccard_off[q], O, &B);
        d.ccard_pos[q] = dupload(P.ccard_pos[q], O, &B);
        d.rank_off[q] = dupload(P.rank_off[q], O, &B);
        d.rank_cnt[q] = dupload(P.rank_cnt[q], O, &B);
        d.rank[q] = dupload(P.rank[q], O, &B);
        d.reach[q] = (float*)dalloc(P.n_rslots[q] * P.nh[q] * sizeof(float), O, &B);
    }
    d.cards = dupload(P.cards, O, &B);
    d.cfv = (float*)dalloc(P.n_cslots * (size_t)P.nh_max * sizeof(float), O, &B);
    d.disc = (float*)dalloc(4 * sizeof(float), O, &B);
    d.iter = (unsigned*)dalloc(sizeof(unsigned), O, &B);
    d.dot = (double*)dalloc(4 * sizeof(double), O, &B);
    CK(cudaMemcpy(d.iter, &E.iteration, sizeof(unsigned), cudaMemcpyHostToDevice));
    E.act = dupload(P.act, O, &B);
    E.edge = dupload(P.edge, O, &B);
    E.fold = dupload(P.fold, O, &B);
    E.show = dupload(P.show, O, &B);
    E.chance = dupload(P.chance, O, &B);
    E.show_smem = (size_t)(4 * P.max_sorted + 53) * sizeof(double);
    if (E.show_smem > 48 * 1024) CK(cudaFuncSetAttribute(k_showdown, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)E.show_smem));

    // arenas
    const size_t esz = E.fmt == kFmtF32 ? 4 : 2;
    for (int q = 0; q < 2; q++) {
        const size_t len = P.arena_len[q];
        E.ar.reg[q] = dalloc(len * esz, O, &B);
        E.ar.str[q] = dalloc(len * esz, O, &B);
        E.ar.pred[q] = E.pcfr ? dalloc(len * esz, O, &B) : nullptr;
        if (E.fmt == kFmtI16) {
            E.ar.rscale[q] = (float*)dalloc(std::max<uint64_t>(P.n_anodes[q], 1) * 4, O, &B);
            E.ar.sscale[q] = (float*)dalloc(std::max<uint64_t>(P.n_anodes[q], 1) * 4, O, &B);
            E.ar.pscale[q] = E.pcfr ? (float*)dalloc(std::max<uint64_t>(P.n_anodes[q], 1) * 4, O, &B) : nullptr;
        }
        for (uint64_t s = 0; s < P.n_anodes[q]; s++) {
            const uint32_t nd = P.anode_id[q][s];
            E.hx[q].push_back({sp.tree.data_off[nd], P.anode_off[q][s], sp.tree.nchild[nd], (uint32_t)s});
        }
        E.xnodes[q] = dupload(E.hx[q], O, &B);
    }
    E.staging_len = std::max<uint64_t>(std::max(sp.tree.data_size[0], sp.tree.data_size[1]), 1);
    E.staging = (float*)dalloc(E.staging_len * sizeof(float), O, &B);
    CK(cudaMallocHost(&E.pinned, E.staging_len * sizeof(float)));
    CK(cudaMallocHost(&E.h_dot, 4 * sizeof(double)));

    // upload arenas: quants directly when host and device are both 16-bit, else via f32 (+ encode)
    std::vector<float> img(E.staging_len);
    for (int q = 0; q < 2; q++) {
        const int nh = P.nh[q];
        const unsigned nb = (unsigned)P.n_anodes[q];
        if (!nb) continue;
        for (int which = 0; which < 3; which++) {
            if (which == kPreds && !E.pcfr) continue;
            void* dst = which == kRegrets ? E.ar.reg[q] : which == kStrategy ? E.ar.str[q] : E.ar.pred[q];
            const Arena* ha = which == kRegrets ? &host.regrets[q] : which == kStrategy ? &host.strat[q]
                              : (host.have_preds ? &host.preds[q] : nullptr);
            if (!ha) continue;  // predictions start at zero
            if (E.fmt == kFmtI16 && ha->kind != 0) {
                const size_t len = sp.tree.data_size[q];
                if (ha->kind == 1) CK(cudaMemcpy(E.staging, ha->qi.data(), len * 2, cudaMemcpyHostToDevice));
                else CK(cudaMemcpy(E.staging, ha->qu.data(), len * 2, cudaMemcpyHostToDevice));
                k_to_dev<uint16_t><<<nb, kThreads, 0, E.stream>>>((const uint16_t*)E.staging, (uint16_t*)dst, E.xnodes[q], nh);
                std::vector<float> sc(P.n_anodes[q]);
                for (uint64_t s = 0; s < P.n_anodes[q]; s++) sc[s] = ha->scale[P.anode_id[q][s]];
                float* dsc = which == kRegrets ? E.ar.rscale[q] : which == kStrategy ? E.ar.sscale[q] : E.ar.pscale[q];
                CK(cudaMemcpyAsync(dsc, sc.data(), sc.size() * 4, cudaMemcpyHostToDevice, E.stream));
                CK(cudaStreamSynchronize(E.stream));
                continue;
            }
            host.arena_f32(which, q, img.data());
            CK(cudaMemcpy(E.staging, img.data(), sp.tree.data_size[q] * 4, cudaMemcpyHostToDevice));
            if (E.fmt == kFmtF32) {
                k_to_dev<float><<<nb, kThreads, 0, E.stream>>>(E.staging, (float*)dst, E.xnodes[q], nh);
            } else {
                float* dsc = which == kRegrets ? E.ar.rscale[q] : which == kStrategy ? E.ar.sscale[q] : E.ar.pscale[q];
                k_encode<<<nb, kThreads, 0, E.stream>>>(E.staging, dst, dsc, E.xnodes[q], nh, which == kStrategy);
            }
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(E.stream));
        }
    }
    E.upload_locks(host);
    CK(cudaStreamSynchronize(E.stream));
}

GpuEngine::~GpuEngine() = default;

void GpuEngine::iterate(int n) {
    EngineImpl& E = *d_;
    for (int k = 0; k < n; k++) {
        if (!E.g_iter) E.g_iter = E.capture(-1);
        CK(cudaGraphLaunch(E.g_iter, E.stream));
        E.iteration++;
    }
    CK(cudaGetLastError());
}

double GpuEngine::time_iterations(int n) {
    EngineImpl& E = *d_;
    if (!E.g_iter) E.g_iter = E.capture(-1);
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, E.stream));
    for (int k = 0; k < n; k++) {
        CK(cudaGraphLaunch(E.g_iter, E.stream));
        E.iteration++;
    }
    CK(cudaEventRecord(b, E.stream));
    CK(cudaEventSynchronize(b));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

Profile GpuEngine::iterate_profiled() {
    EngineImpl& E = *d_;
    Profile pr;
    std::memset(&pr, 0, sizeof(pr));
    CK(cudaStreamSynchronize(E.stream));
    k_begin_iteration<<<1, 1, 0, E.stream>>>(E.d.iter, E.d.disc, E.algo);
    E.sweep(0, -1, &pr);
    E.sweep(1, -1, &pr);
    CK(cudaStreamSynchronize(E.stream));
    E.iteration++;
    return pr;
}

double GpuEngine::exploitability(const HostSolver& host) {  // best_response.rs:255-287
    EngineImpl& E = *d_;
    const double denom = host.spot->pair_weight_sum();
    if (denom <= 0.0) return NAN;
    const bool raked = host.spot->config.tree.rake_pct > 0.0;
    double br[2], v[2] = {0, 0};
    for (int mode = 0; mode < (raked ? 2 : 1); mode++) {
        if (!E.g_eval[mode]) E.g_eval[mode] = E.capture(mode);
        CK(cudaGraphLaunch(E.g_eval[mode], E.stream));
        CK(cudaStreamSynchronize(E.stream));
        for (int p = 0; p < 2; p++) (mode == 0 ? br[p] : v[p]) = E.h_dot[p] / denom;
    }
    if (raked) return ((br[0] - v[0]) + (br[1] - v[1])) / 2.0;
    return (br[0] + br[1]) / 2.0;
}

void GpuEngine::root_cfv(int p, int mode, float* out) {
    EngineImpl& E = *d_;
    E.sweep(p, mode, nullptr);
    CK(cudaMemcpyAsync(out, E.d.cfv, E.plan.nh[p] * sizeof(float), cudaMemcpyDeviceToHost, E.stream));
    CK(cudaStreamSynchronize(E.stream));
}

void GpuEngine::export_arena(int which, int p, float* out) {
    EngineImpl& E = *d_;
    const Spot& sp = *E.spot;
    const size_t len = sp.tree.data_size[p];
    CK(cudaMemsetAsync(E.staging, 0, E.staging_len * 4, E.stream));
    const unsigned nb = (unsigned)E.plan.n_anodes[p];
    void* src = which == kRegrets ? E.ar.reg[p] : which == kStrategy ? E.ar.str[p] : E.ar.pred[p];
    if (nb && src) {
        if (E.fmt == kFmtF32) {
            k_to_host<float><<<nb, kThreads, 0, E.stream>>>((const float*)src, E.staging, E.xnodes[p], E.plan.nh[p]);
        } else if (which == kStrategy) {
            k_decode_to_host<uint16_t><<<nb, kThreads, 0, E.stream>>>((const uint16_t*)src, E.ar.sscale[p], E.staging,
                                                                       E.xnodes[p], E.plan.nh[p], 65535.0f);
        } else {
            const float* sc = which == kRegrets ? E.ar.rscale[p] : E.ar.pscale[p];
            k_decode_to_host<int16_t><<<nb, kThreads, 0, E.stream>>>((const int16_t*)src, sc, E.staging, E.xnodes[p],
                                                                      E.plan.nh[p], 32767.0f);
        }
        CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(out, E.staging, len * 4, cudaMemcpyDeviceToHost, E.stream));
    CK(cudaStreamSynchronize(E.stream));
}

void GpuEngine::sync_to_cpu(HostSolver& host, bool strategy_only) {  // gpu/mod.rs:845-886
    EngineImpl& E = *d_;
    CK(cudaStreamSynchronize(E.stream));
    const Spot& sp = *E.spot;
    const Tree& t = sp.tree;
    for (int p = 0; p < 2; p++) {
        const int nh = E.plan.nh[p];
        for (int which = strategy_only ? 1 : 0; which < (E.pcfr && !strategy_only ? 3 : 2); which++) {
            Arena& ha = which == kRegrets ? host.regrets[p] : which == kStrategy ? host.strat[p]
                                                             : (host.ensure_preds(), host.preds[p]);
            const unsigned nb = (unsigned)E.plan.n_anodes[p];
            if (!nb) continue;
            void* src = which == kRegrets ? E.ar.reg[p] : which == kStrategy ? E.ar.str[p] : E.ar.pred[p];
            if (E.fmt == kFmtI16 && ha.kind != 0) {
                // 16-bit on both sides: quants and scales move exactly
                k_to_host<uint16_t><<<nb, kThreads, 0, E.stream>>>((const uint16_t*)src, (uint16_t*)E.staging, E.xnodes[p], nh);
                CK(cudaMemcpyAsync(E.pinned, E.staging, t.data_size[p] * 2, cudaMemcpyDeviceToHost, E.stream));
                std::vector<float> sc(E.plan.n_anodes[p]);
                const float* dsc = which == kRegrets ? E.ar.rscale[p] : which == kStrategy ? E.ar.sscale[p] : E.ar.pscale[p];
                CK(cudaMemcpyAsync(sc.data(), dsc, sc.size() * 4, cudaMemcpyDeviceToHost, E.stream));
                CK(cudaStreamSynchronize(E.stream));
                const uint16_t* q = (const uint16_t*)E.pinned;
                for (uint64_t s = 0; s < E.plan.n_anodes[p]; s++) {
                    const uint32_t nd = E.plan.anode_id[p][s];
                    const size_t off = t.data_off[nd], cnt = (size_t)t.nchild[nd] * nh;
                    if (ha.kind == 1) std::memcpy(ha.qi.data() + off, q + off, cnt * 2);
                    else std::memcpy(ha.qu.data() + off, q + off, cnt * 2);
                    ha.scale[nd] = sc[s];
                }
                continue;
            }
            export_arena(which, p, E.pinned);
            for (uint64_t s = 0; s < E.plan.n_anodes[p]; s++) {
                const uint32_t nd = E.plan.anode_id[p][s];
                ha.write(nd, t.data_off[nd], (size_t)t.nchild[nd] * nh, E.pinned + t.data_off[nd]);
            }
        }
    }
    host.iteration = E.iteration;
    if (E.plan.iso_active) host.sym_dirty = true;
}

void GpuEngine::synchronize() { CK(cudaStreamSynchronize(d_->stream)); }
void GpuEngine::update_locks(const HostSolver& host) { d_->upload_locks(host); }
uint32_t GpuEngine::iteration() const { return d_->iteration; }
int GpuEngine::format() const { return d_->fmt; }
const Plan& GpuEngine::plan() const { return d_->plan; }
uint64_t GpuEngine::device_bytes() const { return d_->bytes; }
void GpuEngine::discounts(float* out3) {
    CK(cudaMemcpyAsync(out3, d_->d.disc, 3 * sizeof(float), cudaMemcpyDeviceToHost, d_->stream));
    CK(cudaStreamSynchronize(d_->stream));
}
double GpuEngine::iter_bytes() const {
    // Algorithmic bytes of one iteration: sigma reads of both arenas in both
    // down sweeps, read+write of the traverser's regrets and sums, one
    // opponent-reach read and one cfv write per terminal per traversal.
    const Plan& P = d_->plan;
    const double b = d_->fmt == kFmtF32 ? 4.0 : 2.0;
    const double D = (double)(P.visited_action_elems[0] + P.visited_action_elems[1]);
    double bytes = 2.0 * D * b + 2.0 * D * (b + b) + 2.0 * (double)P.visited_terminals * (P.nh[0] + P.nh[1]) * 4.0;
    if (d_->fmt != kFmtF32) bytes += 8.0 * (double)(P.n_anodes[0] + P.n_anodes[1]) * 2.0;
    return bytes;
}

uint64_t estimate_vram(const Spot& spot) {  // same role as game.rs:365-373, for this engine's layout
    Plan P = build_plan(spot, true);
    uint64_t b = P.n_cslots * (uint64_t)P.nh_max * 4 + P.n_rslots[0] * (uint64_t)P.nh[0] * 4 +
                 P.n_rslots[1] * (uint64_t)P.nh[1] * 4;
    b += (P.arena_len[0] + P.arena_len[1]) * 2 * 4;
    return b + 512ull * 1024 * 1024;
}
bool vram_info_mb(uint64_t* free_mb, uint64_t* total_mb) {
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) return false;
    *free_mb = f / 1000000;
    *total_mb = t / 1000000;
    return true;
}

}  // namespace gtob
