// Batched engine: the CFR iterations of many spots in ONE persistent kernel
// launch per iteration, driven by a (spot, step, node-tile) work queue.
//
// A spot's iteration is a fixed list of steps -- per traverser: the
// iteration's discounts and the root reach, each level of the down sweep,
// every showdown batch, each level of the up sweep (deepest first) -- and a
// step is one to three spans of node records of one kind (the staged
// engine's records: SNode, EdgeItem, ShowBatch, ChanceItem).  Records of one
// step never depend on each other, exactly as the CTAs of one launch of the
// level-synchronous engine don't.
//
// The queue is a table of segments (one span of one step of one spot),
// ordered by step index, then spot, so that the spots' steps interleave.  A
// segment is cut into tickets of `tile` records.  A CTA takes the next
// ticket from a global counter, waits until its spot has finished every
// ticket of its earlier steps (a per-spot counter), runs the ticket's
// records with the staged engine's node functions, and adds one to the
// spot's counter.  A ticket only waits on tickets with smaller numbers, all
// taken by CTAs that are running, so the kernel cannot deadlock whatever its
// grid.  Every wait is bounded (kWaitNs): a wait that gives up sets bit 2 of
// the control word's error field and the abort flag, and every CTA stops at
// its next ticket.
//
// Visibility between CTAs: the producer's threads fence their generic
// stores for the bulk-copy (async) proxy and the CTA's release increments
// the spot counter after a block barrier; the consumer acquires the counter
// and fences for the async proxy before its first bulk copy.  Node records
// in one CTA run back to back in the same dynamic shared memory: each one's
// mbarriers are invalidated and its shared-memory accesses fenced for the
// async proxy before the next record's copies are issued.
//
// The arithmetic is the staged engine's node functions (the chance node's at
// 128 threads instead of 256): per hand in registers, block maxima, and
// exact (integer) terminal sums, so the results are bit-identical to the
// spot's own engine.
#pragma once
#include "cfr_staged.cuh"

namespace gtob {

// 128 threads, the staged node kernels' width: the CTA count per SM is set
// by the largest shared-memory need over the record kinds (a showdown
// batch's), so a narrow CTA keeps the most nodes in flight
constexpr int kBThreads = kSThreads;
// (BatchKind, the record kinds of a ticket: host/plan.hpp)

// One spot as the batched kernel reads it (copied to shared memory when a
// CTA starts a ticket of a spot other than its last one).
struct alignas(16) BSpot {
    Dev d;
    Arenas ar;
    const SNode* snodes;
    const EdgeItem* edge;
    const ShowItem* show;
    const ShowBatch* show_batch;
    const ChanceItem* chance;
    int msort;  // the plan's max_sorted (showdown tables)
    int algo;
};
// One queue segment: `count` records of one kind of one step of one spot,
// starting at record `start` of that kind's array, in tickets of `tile`.
struct alignas(16) BSeg {
    uint32_t first;  // the segment's first ticket
    uint32_t start;
    uint32_t count;
    uint32_t need;   // tickets of this spot in earlier steps: done before any of this segment runs
    uint16_t spot;
    uint8_t kind;    // BatchKind
    uint8_t p;       // traverser (show, chance, up); players whose reach is refreshed (edge: qmask)
    uint16_t tile;
    uint16_t pad0;
    uint32_t pad1, pad2;
};
static_assert(sizeof(BSeg) == 32, "BSeg layout");
// Control words of one launch (zeroed before it): [0] next ticket, [1]
// abort, [2] error bits, [3] unused, [4 + s] tickets spot s has finished.
constexpr int kBCtlHead = 0, kBCtlAbort = 1, kBCtlErr = 2, kBCtlDone = 4;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Thread 0: bounded wait until *cnt >= need.  False when the launch is
// aborting (another CTA gave up) or this wait gave up (abort raised).
__device__ bool b_wait_count(const unsigned* cnt, unsigned need, unsigned* ctl) {
    if (ld_acquire_u32(cnt) >= need) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        __nanosleep(256);
        if (ld_acquire_u32(cnt) >= need) return true;
        if (*(volatile unsigned*)(ctl + kBCtlAbort)) return false;
        if (globaltimer_ns() - t0 > kWaitNs) {
            atomicOr(ctl + kBCtlErr, 4u);
            atomicExch(ctl + kBCtlAbort, 1u);
            return false;
        }
    }
}

template <int FMT>
__device__ __forceinline__ void b_down(const BSpot& S, uint32_t r, unsigned char* sm, int& s_flag) {
    const SNode it = S.snodes[r];
    switch (it.na) {
        case 1: ks_down_node<FMT, 1, kBThreads>(S.d, S.ar, it, 0, sm, s_flag); break;
        case 2: ks_down_node<FMT, 2, kBThreads>(S.d, S.ar, it, 0, sm, s_flag); break;
        case 3: ks_down_node<FMT, 3, kBThreads>(S.d, S.ar, it, 0, sm, s_flag); break;
        default: ks_down_node<FMT, 4, kBThreads>(S.d, S.ar, it, 0, sm, s_flag); break;
    }
}
template <int FMT, bool MINE>
__device__ __forceinline__ void b_up(const BSpot& S, uint32_t r, int p, unsigned char* sm, UpSharedT<kBThreads>& us) {
    const SNode it = S.snodes[r];
    switch (it.na) {
        case 1: ks_up_node<FMT, 0, 1, MINE, kBThreads>(S.d, S.ar, it, p, 0, sm, us); break;
        case 2: ks_up_node<FMT, 0, 2, MINE, kBThreads>(S.d, S.ar, it, p, 0, sm, us); break;
        case 3: ks_up_node<FMT, 0, 3, MINE, kBThreads>(S.d, S.ar, it, p, 0, sm, us); break;
        default: ks_up_node<FMT, 0, 4, MINE, kBThreads>(S.d, S.ar, it, p, 0, sm, us); break;
    }
}

// One CFR iteration of every spot of the queue.  ctl: the launch's control
// words (zeroed before the launch).
template <int FMT>
__global__ void __launch_bounds__(kBThreads, 4) kb_iterate(const BSpot* spots, const BSeg* segs, int nseg,
                                                        unsigned nticket, unsigned* ctl) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ BSpot s_spot;
    __shared__ UpSharedT<kBThreads> us;
    __shared__ ShowShared<kBThreads> ss;
    __shared__ long long s_cw[kBThreads / 32];
    __shared__ int s_flag;
    __shared__ unsigned s_t, s_seg, s_go;
    __shared__ int s_have;  // the spot in s_spot (-1: none yet)
    if (threadIdx.x == 0) s_have = -1;
    for (;;) {
        if (threadIdx.x == 0) {
            s_go = 0;
            const unsigned t = *(volatile unsigned*)(ctl + kBCtlAbort) ? nticket : atomicAdd(ctl + kBCtlHead, 1u);
            s_t = t;
            if (t < nticket) {
                int lo = 0, hi = nseg - 1;  // the last segment whose first ticket is <= t
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (segs[mid].first <= t) lo = mid;
                    else hi = mid - 1;
                }
                s_seg = (unsigned)lo;
                const BSeg& sg = segs[lo];
                if (b_wait_count(ctl + kBCtlDone + sg.spot, sg.need, ctl)) {
                    fence_async_global();  // the spot's earlier writes, seen by this CTA's bulk copies
                    s_go = 1;
                }
            }
        }
        __syncthreads();
        if (!s_go) break;
        const BSeg sg = segs[s_seg];
        if (s_have != (int)sg.spot) {  // this spot's record into shared memory
            const int4* src = (const int4*)(spots + sg.spot);
            int4* dst = (int4*)&s_spot;
            for (unsigned k = threadIdx.x; k < sizeof(BSpot) / 16; k += kBThreads) dst[k] = src[k];
            __syncthreads();
            if (threadIdx.x == 0) s_have = (int)sg.spot;
        }
        const BSpot& S = s_spot;
        const uint32_t r0 = sg.start + (s_t - sg.first) * (uint32_t)sg.tile;
        const uint32_t r1 = min(r0 + (uint32_t)sg.tile, sg.start + sg.count);
        const int p = sg.p;
        for (uint32_t r = r0; r < r1; r++) {
            switch (sg.kind) {
                case kBBegin:
                    if (threadIdx.x == 0) begin_iteration(S.d.iter, S.d.disc, S.algo);
                    break;
                case kBRoot:
                    for (int q = 0; q < 2; q++)
                        for (int i = threadIdx.x; i < S.d.nh[q]; i += kBThreads) S.d.reach[q][i] = S.d.w[q][i];
                    break;
                case kBDown: b_down<FMT>(S, r, sm, s_flag); break;
                case kBEdge: edge_down(S.d, S.edge[r], p); break;
                case kBShow: show_batch_run<kBThreads>(S.d, S.show, S.show_batch[r], p, S.msort, sm, ss); break;
                case kBChance: chance_node<long long, kBThreads>(S.d, S.chance[r], p, (double*)sm, s_cw); break;
                case kBUpMine: b_up<FMT, true>(S, r, p, sm, us); break;
                default: b_up<FMT, false>(S, r, p, sm, us); break;
            }
            // the next record reuses the shared memory: generic accesses
            // ordered before its bulk copies, this record's barriers retired;
            // a copy that failed (the spot's error word) stops the launch
            fence_async_shared();
            const bool bad = __syncthreads_or(threadIdx.x == 0 && *(volatile unsigned*)S.d.err != 0u);
            if (threadIdx.x == 0) {
                if (sg.kind == kBDown || sg.kind == kBUpMine || sg.kind == kBUpOpp) mbar_inval((uint64_t*)sm);
                if (sg.kind == kBShow) {
                    mbar_inval((uint64_t*)sm);
                    mbar_inval((uint64_t*)sm + 1);
                }
                if (bad) atomicExch(ctl + kBCtlAbort, 1u);
            }
            if (bad) break;
        }
        fence_async_global();  // this ticket's stores, for the bulk copies of later tickets
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(ctl + kBCtlDone + sg.spot, 1u);
        }
    }
}

}  // namespace gtob
