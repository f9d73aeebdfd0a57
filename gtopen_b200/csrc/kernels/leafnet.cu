// The turn-leaf value network's kernels: one tcgen05 BF16 matrix product
// with fused epilogues, and the elementwise pieces of training around it
// (packing, transposes, masked squared error, bias gradients, Adam).
//
// k_gemm_tn<BN>, one 128 x BN output tile per CTA (BN = 256 where N is a
// multiple of 256, else 128), 4 warps:
//   * warp 0 lane 0 streams 128 x 64 tiles of A and BN x 64 tiles of B into a
//     4-stage ring of shared memory with TMA (cp.async.bulk.tensor, 128-byte
//     swizzle), one mbarrier per stage counting the bytes;
//   * warp 1 lane 0 issues tcgen05.mma (kind::f16, BF16 in, FP32 accumulate,
//     M = 128, N = BN) into a BN-column tensor-memory accumulator, four K=16
//     steps per stage, and frees each stage with tcgen05.commit on its
//     "empty" mbarrier;
//   * then all four warps read their 32 accumulator lanes with tcgen05.ld and
//     apply the epilogue (bias, pre-activation store, GELU' product, GELU,
//     f32 / bf16 stores) straight to global memory.
// Every mbarrier wait is bounded (2 s of %globaltimer): a wait that gives up
// sets an error bit the host reads, and the tile is skipped; the tensor
// memory is always freed.
#include "leafnet.hpp"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>

#include "../host/core.hpp"

namespace gtob {

#define LCK(x)                                                                                          \
    do {                                                                                                \
        cudaError_t e_ = (x);                                                                           \
        if (e_ != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(e_) + " at " #x); \
    } while (0)

namespace {

constexpr int kBM = 128, kBK = 64, kStages = 4;
constexpr int kGemmThreads = 128;
constexpr uint32_t kTileABytes = kBM * kBK * 2;
constexpr unsigned long long kNetWaitNs = 2000000000ull;
constexpr unsigned kErrGemmWait = 16u;
// A 128 x BN output tile (BN = 128 or 256: TMEM columns, B rows per stage).
template <int BN>
struct TileCfg {
    static constexpr uint32_t kTileB = BN * kBK * 2;
    static constexpr uint32_t kStage = kTileABytes + kTileB;
    static constexpr size_t kSmem = (size_t)kStages * kStage + 1024;  // + room to align the ring to 1 KiB
    // instruction descriptor: kind::f16, D f32 (bits 4-5 = 1), A and B bf16
    // (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
    static constexpr uint32_t kIdesc =
        (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
};

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void bar_init(uint64_t* b, unsigned n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* b, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}
__device__ __noinline__ bool bar_wait(uint64_t* b, unsigned parity) {
    if (bar_try(b, parity)) return true;
    const unsigned long long t0 = gtimer();
    while (!bar_try(b, parity))
        if (gtimer() - t0 > kNetWaitNs) return false;
    return true;
}
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            su32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(su32(bar))
        : "memory");
}
__device__ __forceinline__ void tm_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tm_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// shared-memory matrix descriptor of a K-major tile of 128-byte rows in the
// 128-byte swizzle (8-row atoms of 1 KiB): start >> 4, leading offset 16 B,
// stride offset 1 KiB between 8-row groups, descriptor version 1, swizzle 2
__device__ __forceinline__ uint64_t sw128_desc(const void* p) {
    const uint32_t a = su32(p);
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) |
           ((uint64_t)2 << 61);
}
__device__ __forceinline__ void tm_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void tm_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}
// 16 consecutive f32 columns of this thread's accumulator lane
__device__ __forceinline__ void tm_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    // the registers are not valid before the wait: tie them to it
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    return cdf + z * (expf(-0.5f * z * z) * 0.39894228040143268f);
}

__device__ __forceinline__ void epilogue16(const GemmEpilogue& e, int row, int col, float* v) {
    if (e.bias) {
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] += e.bias[col + i];
    }
    if (e.pre) {
        float4* o = (float4*)(e.pre + (size_t)row * e.ld_pre + col);
#pragma unroll
        for (int i = 0; i < 4; i++) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    }
    if (e.gmul) {
        const float4* g = (const float4*)(e.gmul + (size_t)row * e.ld_gmul + col);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float4 z = g[i];
            v[4 * i] *= gelu_grad(z.x);
            v[4 * i + 1] *= gelu_grad(z.y);
            v[4 * i + 2] *= gelu_grad(z.z);
            v[4 * i + 3] *= gelu_grad(z.w);
        }
    }
    if (e.gelu) {
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = gelu_f(v[i]);
    }
    if (e.out_f32) {
        float4* o = (float4*)(e.out_f32 + (size_t)row * e.ld_f32 + col);
#pragma unroll
        for (int i = 0; i < 4; i++) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    }
    if (e.out_bf16) {
        __nv_bfloat162 h[8];
#pragma unroll
        for (int i = 0; i < 8; i++) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        uint4* o = (uint4*)(e.out_bf16 + (size_t)row * e.ld_bf16 + col);
        o[0] = *(const uint4*)&h[0];
        o[1] = *(const uint4*)&h[4];
    }
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm_tn(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int K, GemmEpilogue e,
              unsigned* err) {
    extern __shared__ uint8_t dsm[];
    uint8_t* ring = dsm + ((1024u - (su32(dsm) & 1023u)) & 1023u);  // 1 KiB aligned: the swizzle atoms
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done;
    __shared__ uint32_t tbase;
    __shared__ int aborted, issued;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    using T = TileCfg<BN>;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN, nk = K / kBK;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            bar_init(&full[s], 1);
            bar_init(&empty[s], 1);
        }
        bar_init(&done, 1);
        aborted = 0;
        issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tbase)),
                     "r"((uint32_t)BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tm_fence_before();
    __syncthreads();
    tm_fence_after();
    const uint32_t tmem = tbase;
    if (warp == 0 && lane == 0) {  // producer
        int kb = 0;
        for (; kb < nk; kb++) {
            const int s = kb % kStages;
            if (kb >= kStages && !bar_wait(&empty[s], ((kb / kStages) & 1) ^ 1)) {
                atomicOr(err, kErrGemmWait);
                aborted = 1;
                break;
            }
            uint8_t* sa = ring + (size_t)s * T::kStage;
            bar_expect_tx(&full[s], T::kStage);
            tma_2d(sa, &ta, kb * kBK, m0, &full[s]);
            tma_2d(sa + kTileABytes, &tb, kb * kBK, n0, &full[s]);
        }
        issued = kb;
    } else if (warp == 1 && lane == 0) {  // MMA issuer
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb % kStages;
            if (!bar_wait(&full[s], (kb / kStages) & 1)) {
                atomicOr(err, kErrGemmWait);
                aborted = 1;
                break;
            }
            tm_fence_after();
            const uint8_t* sa = ring + (size_t)s * T::kStage;
            const uint64_t da = sw128_desc(sa), db = sw128_desc(sa + kTileABytes);
#pragma unroll
            for (int k = 0; k < kBK / 16; k++) tm_mma(tmem, da + 2 * k, db + 2 * k, T::kIdesc, (kb | k) ? 1u : 0u);
            tm_commit(&empty[s]);  // the stage is free once these products have read it
        }
        tm_commit(&done);  // arrives when every product issued above has finished
    }
    __syncwarp();
    const bool ok = bar_wait(&done, 0);
    const int good = __syncthreads_and(ok ? 1 : 0) && !aborted;
    if (!ok && threadIdx.x == 0) atomicOr(err, kErrGemmWait);
    if (!good) {
        // Abort: let the work already started finish before the CTA frees
        // its TMEM and exits -- a second bounded wait for the products in
        // flight (done arrives once every issued product has completed; the
        // MMA thread commits it on its error path too), and, on the
        // producer, for the tile loads it issued that no product waited
        // for (at most the last kStages: a load is only issued once the
        // product kStages before it has read its stage).
        if (!ok) bar_wait(&done, 0);
        if (warp == 0 && lane == 0)
            for (int kb = issued > kStages ? issued - kStages : 0; kb < issued; kb++)
                bar_wait(&full[kb % kStages], (kb / kStages) & 1);
    }
    tm_fence_after();
    if (good) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c = 0; c < BN; c += 16) {
            float v[16];
            tm_ld16(lane_base + (uint32_t)c, v);
            epilogue16(e, row, n0 + c, v);
        }
    }
    tm_fence_before();
    __syncthreads();
    if (warp == 0) {
        tm_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN)
                     : "memory");
    }
}

// ---------------------------------------------------------------- training pieces
// out[c * R + r] = in[r * C + c] (bf16), 32 x 32 tiles through shared memory
__global__ void k_transpose(const __nv_bfloat16* __restrict__ in, int R, int C, __nv_bfloat16* __restrict__ out) {
    __shared__ __nv_bfloat16 t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) t[j][threadIdx.x] = in[(size_t)(r0 + j) * C + c0 + threadIdx.x];
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) out[(size_t)(c0 + j) * R + r0 + threadIdx.x] = t[threadIdx.x][j];
}
// rows of a row-major f32 table (row idx[i] of width w) into padded buffers:
// bf16 (x) or f32 (y); padding rows and columns zero
__global__ void k_gather_rows_bf16(const float* __restrict__ src, const int* __restrict__ idx, int n, int w, int wp,
                                   __nv_bfloat16* __restrict__ dst) {
    const int r = blockIdx.x;
    for (int c = threadIdx.x; c < wp; c += blockDim.x) {
        const float v = r < n && c < w ? src[(size_t)idx[r] * w + c] : 0.0f;
        dst[(size_t)r * wp + c] = __float2bfloat16_rn(v);
    }
}
__global__ void k_gather_rows_f32(const float* __restrict__ src, const int* __restrict__ idx, int n, int w, int wp,
                                  float* __restrict__ dst) {
    const int r = blockIdx.x;
    for (int c = threadIdx.x; c < wp; c += blockDim.x)
        dst[(size_t)r * wp + c] = r < n && c < w ? src[(size_t)idx[r] * w + c] : 0.0f;
}
// masked squared error, averaged over n * w entries: dy = d loss / d y (f32
// and bf16), loss accumulated in f64
__global__ void k_loss(const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ m,
                       size_t total, float inv, float* __restrict__ dy, __nv_bfloat16* __restrict__ dyb,
                       double* loss) {
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const float d = (y[i] - t[i]) * m[i];
        const float g = 2.0f * d * inv;
        dy[i] = g;
        dyb[i] = __float2bfloat16_rn(g);
        acc += (double)d * d;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += part[w];
        atomicAdd(loss, s * (double)inv);
    }
}
// out[c] = sum over rows of g[r * N + c]
__global__ void k_colsum(const float* __restrict__ g, int rows, int N, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    float s = 0.0f;
    for (int r = 0; r < rows; r++) s += g[(size_t)r * N + c];
    out[c] = s;
}
// Adam on the f32 masters; refreshes the bf16 copy (mask: padded entries
// stay zero)
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, const uint8_t* __restrict__ live, size_t n, float lr, float b1, float b2,
                       float eps, float bc1, float bc2, __nv_bfloat16* __restrict__ wb) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (live && !live[i]) continue;
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float step = lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] -= step;
        if (wb) wb[i] = __float2bfloat16_rn(w[i]);
    }
}
__global__ void k_to_bf16(const float* __restrict__ in, size_t n, __nv_bfloat16* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = __float2bfloat16_rn(in[i]);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    // resolved once (a function-local static: thread-safe; a failed lookup is retried)
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        LCK(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) throw Error("cuda: cuTensorMapEncodeTiled is not available");
        return (PFN_cuTensorMapEncodeTiled_v12000)p;
    }();
    return fn;
}
// a row-major bf16 matrix (rows x inner) read in 64 x box_rows boxes, 128-byte swizzle
CUtensorMap tile_map(const void* base, uint64_t inner, uint64_t rows, uint32_t box_rows) {
    CUtensorMap m;
    cuuint64_t dims[2] = {inner, rows};
    cuuint64_t strides[1] = {inner * 2};
    cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                                   box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error("cuda: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}
template <class T>
T* dnew(size_t n) {
    void* p = nullptr;
    LCK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    LCK(cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T)));
    return (T*)p;
}
int pad128(int x) { return (x + 127) / 128 * 128; }
int grid_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }
uint64_t xs_next(uint64_t& s) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
}

}  // namespace

template <int BN>
static void launch_gemm(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, const GemmEpilogue& e,
                        unsigned* err, cudaStream_t s) {
    const CUtensorMap ta = tile_map(A, (uint64_t)K, (uint64_t)M, kBM);
    const CUtensorMap tb = tile_map(B, (uint64_t)K, (uint64_t)N, (uint32_t)BN);
    // once per device, so that a captured stream makes no attribute calls
    static std::atomic<uint64_t> prepared{0};
    int dev = 0;
    LCK(cudaGetDevice(&dev));
    if (dev >= 64 || !((prepared.load() >> dev) & 1u)) {
        LCK(cudaFuncSetAttribute(k_gemm_tn<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TileCfg<BN>::kSmem));
        if (dev < 64) prepared.fetch_or(uint64_t(1) << dev);
    }
    k_gemm_tn<BN><<<dim3(N / BN, M / kBM), kGemmThreads, TileCfg<BN>::kSmem, s>>>(ta, tb, K, e, err);
    LCK(cudaGetLastError());
}

void gemm_bf16_tn(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, const GemmEpilogue& e,
                  unsigned* err, cudaStream_t s) {
    if (M <= 0 || N <= 0 || K <= 0 || M % kBM || N % 128 || K % kBK)
        throw Error("invalid argument: matrix product shape (M, N multiples of 128, K of 64)");
    // 128 x 256 tiles where N allows (twice the work per instruction and per
    // tile, half the tiles), else 128 x 128
    if (N % 256 == 0) launch_gemm<256>(A, B, M, N, K, e, err, s);
    else launch_gemm<128>(A, B, M, N, K, e, err, s);
}

double gemm_time_ms(int m, int n, int k, int reps) {
    __nv_bfloat16* a = dnew<__nv_bfloat16>((size_t)m * k);
    __nv_bfloat16* b = dnew<__nv_bfloat16>((size_t)n * k);
    float* c = dnew<float>((size_t)m * n);
    unsigned* err = dnew<unsigned>(1);
    cudaStream_t s;
    cudaEvent_t e0, e1;
    LCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    LCK(cudaEventCreate(&e0));
    LCK(cudaEventCreate(&e1));
    GemmEpilogue ep;
    ep.out_f32 = c;
    ep.ld_f32 = n;
    gemm_bf16_tn(a, b, m, n, k, ep, err, s);  // warm-up (and the attribute call)
    LCK(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; r++) gemm_bf16_tn(a, b, m, n, k, ep, err, s);
    LCK(cudaEventRecord(e1, s));
    LCK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    LCK(cudaEventElapsedTime(&ms, e0, e1));
    unsigned e = 0;
    LCK(cudaMemcpy(&e, err, sizeof(e), cudaMemcpyDeviceToHost));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    for (void* p : {(void*)a, (void*)b, (void*)c, (void*)err}) cudaFree(p);
    if (e) throw Error("timeout: a tensor-core matrix product's wait gave up");
    return (double)ms / reps;
}

// ---------------------------------------------------------------- LeafNet
struct LeafNet::Layer {
    int in = 0, out = 0, in_p = 0, out_p = 0;
    float *w = nullptr, *b = nullptr, *gw = nullptr, *gb = nullptr, *mw = nullptr, *vw = nullptr, *mb = nullptr,
          *vb = nullptr;
    uint8_t* live = nullptr;  // 1 for the unpadded weights
    __nv_bfloat16 *wb = nullptr, *wt = nullptr;
    // activations for rows_cap rows (hidden layers): pre-activation, output,
    // its transpose, and the gradient of the pre-activation (f32, bf16, transposed)
    float *z = nullptr, *dz = nullptr;
    __nv_bfloat16 *h = nullptr, *ht = nullptr, *dzb = nullptr, *dzt = nullptr;
    void free_acts() {
        for (void* p : {(void*)z, (void*)dz, (void*)h, (void*)ht, (void*)dzb, (void*)dzt}) cudaFree(p);
        z = dz = nullptr;
        h = ht = dzb = dzt = nullptr;
    }
    ~Layer() {
        free_acts();
        for (void* p : {(void*)w, (void*)b, (void*)gw, (void*)gb, (void*)mw, (void*)vw, (void*)mb, (void*)vb,
                        (void*)live, (void*)wb, (void*)wt})
            cudaFree(p);
    }
};

LeafNet::LeafNet(const LeafNetDims& d, uint64_t seed) : d_(d) {
    if (d.din <= 0 || d.dh <= 0 || d.nhidden <= 0 || d.dout <= 0 || d.nhidden > 8)
        throw Error("invalid argument: network dimensions");
    din_p_ = pad128(d.din);
    dh_p_ = pad128(d.dh);
    dout_p_ = pad128(d.dout);
    LCK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    err_ = dnew<unsigned>(1);
    loss_ = dnew<double>(1);
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 0x2545F4914F6CDD1Dull;
    if (!s) s = 1;
    for (int l = 0; l <= d.nhidden; l++) {
        auto L = std::make_unique<Layer>();
        L->in = l == 0 ? d.din : d.dh;
        L->in_p = l == 0 ? din_p_ : dh_p_;
        L->out = l == d.nhidden ? d.dout : d.dh;
        L->out_p = l == d.nhidden ? dout_p_ : dh_p_;
        const size_t nw = (size_t)L->out_p * L->in_p;
        for (float** p : {&L->w, &L->gw, &L->mw, &L->vw}) *p = dnew<float>(nw);
        for (float** p : {&L->b, &L->gb, &L->mb, &L->vb}) *p = dnew<float>(L->out_p);
        L->live = dnew<uint8_t>(nw);
        L->wb = dnew<__nv_bfloat16>(nw);
        L->wt = dnew<__nv_bfloat16>(nw);
        // uniform(-a, a) with a = sqrt(3 / fan_in) (unit variance through
        // the layer for unit-variance inputs); the output layer 10x smaller
        const float a = std::sqrt(3.0f / (float)L->in) * (l == d.nhidden ? 0.1f : 1.0f);
        std::vector<float> w(nw, 0.0f);
        std::vector<uint8_t> live(nw, 0);
        for (int o = 0; o < L->out; o++)
            for (int i = 0; i < L->in; i++) {
                const double u = (double)(xs_next(s) >> 11) * (1.0 / 9007199254740992.0);
                w[(size_t)o * L->in_p + i] = (float)((2.0 * u - 1.0) * a);
                live[(size_t)o * L->in_p + i] = 1;
            }
        LCK(cudaMemcpy(L->w, w.data(), nw * 4, cudaMemcpyHostToDevice));
        LCK(cudaMemcpy(L->live, live.data(), nw, cudaMemcpyHostToDevice));
        L_.push_back(std::move(L));
    }
    for (int l = 0; l < layers(); l++) {
        Layer& L = *L_[l];
        const size_t nw = (size_t)L.out_p * L.in_p;
        k_to_bf16<<<grid_for(nw), 256, 0, stream_>>>(L.w, nw, L.wb);
        k_transpose<<<dim3(L.in_p / 32, L.out_p / 32), dim3(32, 8), 0, stream_>>>(L.wb, L.out_p, L.in_p, L.wt);
    }
    check(stream_);
}

LeafNet::~LeafNet() {
    if (stream_) cudaStreamSynchronize(stream_);
    L_.clear();
    for (void* p : {(void*)x_, (void*)xt_, (void*)dyb_, (void*)dyt_, (void*)y_, (void*)dy_, (void*)t_, (void*)m_,
                    (void*)loss_, (void*)err_})
        cudaFree(p);
    if (stream_) cudaStreamDestroy(stream_);
}

void LeafNet::check(cudaStream_t s) {
    LCK(cudaStreamSynchronize(s));
    unsigned e = 0;
    LCK(cudaMemcpy(&e, err_, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) {
        LCK(cudaMemset(err_, 0, sizeof(unsigned)));
        throw Error("timeout: a tensor-core matrix product's wait gave up");
    }
}

void LeafNet::ensure_rows(int rows_pad) {
    if (rows_pad <= rows_cap_) return;
    LCK(cudaStreamSynchronize(stream_));
    for (void* p : {(void*)x_, (void*)xt_, (void*)dyb_, (void*)dyt_, (void*)y_, (void*)dy_, (void*)t_, (void*)m_})
        cudaFree(p);
    const size_t r = (size_t)rows_pad;
    x_ = dnew<__nv_bfloat16>(r * din_p_);
    xt_ = dnew<__nv_bfloat16>(r * din_p_);
    y_ = dnew<float>(r * dout_p_);
    dy_ = dnew<float>(r * dout_p_);
    t_ = dnew<float>(r * dout_p_);
    m_ = dnew<float>(r * dout_p_);
    dyb_ = dnew<__nv_bfloat16>(r * dout_p_);
    dyt_ = dnew<__nv_bfloat16>(r * dout_p_);
    for (int l = 0; l < d_.nhidden; l++) {
        Layer& L = *L_[l];
        L.free_acts();
        const size_t n = r * L.out_p;
        L.z = dnew<float>(n);
        L.dz = dnew<float>(n);
        L.h = dnew<__nv_bfloat16>(n);
        L.ht = dnew<__nv_bfloat16>(n);
        L.dzb = dnew<__nv_bfloat16>(n);
        L.dzt = dnew<__nv_bfloat16>(n);
    }
    rows_cap_ = rows_pad;
}

void LeafNet::forward(const __nv_bfloat16* x, int rows_pad, float* y, bool keep, cudaStream_t s) {
    const __nv_bfloat16* in = x;
    for (int l = 0; l < d_.nhidden; l++) {
        Layer& L = *L_[l];
        GemmEpilogue e;
        e.bias = L.b;
        if (keep) {
            e.pre = L.z;
            e.ld_pre = L.out_p;
        }
        e.gelu = true;
        e.out_bf16 = L.h;
        e.ld_bf16 = L.out_p;
        gemm_bf16_tn(in, L.wb, rows_pad, L.out_p, L.in_p, e, err_, s);
        launches_++;
        in = L.h;
    }
    Layer& O = *L_[d_.nhidden];
    GemmEpilogue e;
    e.bias = O.b;
    e.out_f32 = y;
    e.ld_f32 = O.out_p;
    gemm_bf16_tn(in, O.wb, rows_pad, O.out_p, O.in_p, e, err_, s);
    launches_++;
}

double LeafNet::backward(const float* t, const float* mask, int rows_pad, int rows, cudaStream_t s) {
    const size_t total = (size_t)rows_pad * dout_p_;
    LCK(cudaMemsetAsync(loss_, 0, sizeof(double), s));
    const float inv = 1.0f / (float)((double)rows * d_.dout);  // the mean over the real rows' entries
    k_loss<<<grid_for(total), 256, 0, s>>>(y_, t, mask, total, inv, dy_, dyb_, loss_);
    launches_++;
    for (int l = d_.nhidden; l >= 0; l--) {
        Layer& L = *L_[l];
        const __nv_bfloat16* gb16 = l == d_.nhidden ? dyb_ : L.dzb;  // d loss / d (this layer's pre-activation)
        const float* g32 = l == d_.nhidden ? dy_ : L.dz;
        __nv_bfloat16* gt = l == d_.nhidden ? dyt_ : L.dzt;
        const __nv_bfloat16* in = l == 0 ? x_ : L_[l - 1]->h;
        __nv_bfloat16* in_t = l == 0 ? xt_ : L_[l - 1]->ht;
        k_transpose<<<dim3(L.out_p / 32, rows_pad / 32), dim3(32, 8), 0, s>>>(gb16, rows_pad, L.out_p, gt);
        k_transpose<<<dim3(L.in_p / 32, rows_pad / 32), dim3(32, 8), 0, s>>>(in, rows_pad, L.in_p, in_t);
        GemmEpilogue ew;
        ew.out_f32 = L.gw;
        ew.ld_f32 = L.in_p;
        gemm_bf16_tn(gt, in_t, L.out_p, L.in_p, rows_pad, ew, err_, s);  // dW = G^T X
        k_colsum<<<(L.out_p + 127) / 128, 128, 0, s>>>(g32, rows_pad, L.out_p, L.gb);
        launches_ += 4;
        if (l > 0) {
            Layer& P = *L_[l - 1];
            GemmEpilogue ex;
            ex.gmul = P.z;
            ex.ld_gmul = P.out_p;
            ex.out_f32 = P.dz;
            ex.ld_f32 = P.out_p;
            ex.out_bf16 = P.dzb;
            ex.ld_bf16 = P.out_p;
            gemm_bf16_tn(gb16, L.wt, rows_pad, L.in_p, L.out_p, ex, err_, s);  // dZ_prev = (G W) * gelu'(Z_prev)
            launches_++;
        }
    }
    double loss = 0.0;
    LCK(cudaMemcpyAsync(&loss, loss_, sizeof(double), cudaMemcpyDeviceToHost, s));
    check(s);
    return loss;
}

void LeafNet::adam(float lr, int step, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float bc1 = (float)(1.0 - std::pow((double)b1, step)), bc2 = (float)(1.0 - std::pow((double)b2, step));
    for (int l = 0; l < layers(); l++) {
        Layer& L = *L_[l];
        const size_t nw = (size_t)L.out_p * L.in_p;
        k_adam<<<grid_for(nw), 256, 0, s>>>(L.w, L.gw, L.mw, L.vw, L.live, nw, lr, b1, b2, eps, bc1, bc2, L.wb);
        k_adam<<<grid_for(L.out), 256, 0, s>>>(L.b, L.gb, L.mb, L.vb, nullptr, (size_t)L.out, lr, b1, b2, eps, bc1,
                                               bc2, nullptr);
        k_transpose<<<dim3(L.in_p / 32, L.out_p / 32), dim3(32, 8), 0, s>>>(L.wb, L.out_p, L.in_p, L.wt);
        launches_ += 3;
    }
}

void LeafNet::get_params(int l, float* w, float* b) const {
    if (l < 0 || l >= layers()) throw Error("invalid argument: layer");
    const Layer& L = *L_[l];
    LCK(cudaStreamSynchronize(stream_));
    if (w) LCK(cudaMemcpy2D(w, L.in * 4, L.w, L.in_p * 4, L.in * 4, L.out, cudaMemcpyDeviceToHost));
    if (b) LCK(cudaMemcpy(b, L.b, L.out * 4, cudaMemcpyDeviceToHost));
}
void LeafNet::get_grads(int l, float* w, float* b) const {
    if (l < 0 || l >= layers()) throw Error("invalid argument: layer");
    const Layer& L = *L_[l];
    LCK(cudaStreamSynchronize(stream_));
    if (w) LCK(cudaMemcpy2D(w, L.in * 4, L.gw, L.in_p * 4, L.in * 4, L.out, cudaMemcpyDeviceToHost));
    if (b) LCK(cudaMemcpy(b, L.gb, L.out * 4, cudaMemcpyDeviceToHost));
}
void LeafNet::set_params(int l, const float* w, const float* b) {
    if (l < 0 || l >= layers()) throw Error("invalid argument: layer");
    Layer& L = *L_[l];
    LCK(cudaStreamSynchronize(stream_));
    if (w) LCK(cudaMemcpy2D(L.w, L.in_p * 4, w, L.in * 4, L.in * 4, L.out, cudaMemcpyHostToDevice));
    if (b) LCK(cudaMemcpy(L.b, b, L.out * 4, cudaMemcpyHostToDevice));
    const size_t nw = (size_t)L.out_p * L.in_p;
    k_to_bf16<<<grid_for(nw), 256, 0, stream_>>>(L.w, nw, L.wb);
    k_transpose<<<dim3(L.in_p / 32, L.out_p / 32), dim3(32, 8), 0, stream_>>>(L.wb, L.out_p, L.in_p, L.wt);
    check(stream_);
}

void LeafNet::forward_device(const __nv_bfloat16* x, int rows_pad, float* y, cudaStream_t s) {
    if (rows_pad % 128) throw Error("invalid argument: rows not padded to 128");
    ensure_rows(rows_pad);
    forward(x, rows_pad, y, false, s);
}

namespace {
// a device buffer freed when its scope ends, on error paths too
template <class T>
struct DevBuf {
    T* p = nullptr;
    explicit DevBuf(size_t n) : p(dnew<T>(n)) {}
    ~DevBuf() { cudaFree(p); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};
// host rows -> device table (n x w f32) once per call
struct DevTable {
    DevBuf<float> buf;
    float* p;
    DevTable(const float* h, size_t n) : buf(n), p(buf.p) { LCK(cudaMemcpy(p, h, n * 4, cudaMemcpyHostToDevice)); }
};
}  // namespace

void LeafNet::forward_host(const float* x, int rows, float* y) {
    if (rows <= 0) return;
    const int rp = pad128(rows);
    ensure_rows(rp);
    DevTable X(x, (size_t)rows * d_.din);
    std::vector<int> idx(rows);
    std::iota(idx.begin(), idx.end(), 0);
    DevBuf<int> idx_buf(rows);
    int* didx = idx_buf.p;
    LCK(cudaMemcpy(didx, idx.data(), rows * 4, cudaMemcpyHostToDevice));
    k_gather_rows_bf16<<<rp, 256, 0, stream_>>>(X.p, didx, rows, d_.din, din_p_, x_);
    forward(x_, rp, y_, false, stream_);
    check(stream_);
    LCK(cudaMemcpy2D(y, d_.dout * 4, y_, dout_p_ * 4, d_.dout * 4, rows, cudaMemcpyDeviceToHost));
}

double LeafNet::gradients_host(const float* x, const float* t, const float* mask, int rows) {
    if (rows <= 0) throw Error("invalid argument: rows");
    const int rp = pad128(rows);
    ensure_rows(rp);
    DevTable X(x, (size_t)rows * d_.din), T(t, (size_t)rows * d_.dout), M(mask, (size_t)rows * d_.dout);
    std::vector<int> idx(rows);
    std::iota(idx.begin(), idx.end(), 0);
    DevBuf<int> idx_buf(rows);
    int* didx = idx_buf.p;
    LCK(cudaMemcpy(didx, idx.data(), rows * 4, cudaMemcpyHostToDevice));
    k_gather_rows_bf16<<<rp, 256, 0, stream_>>>(X.p, didx, rows, d_.din, din_p_, x_);
    k_gather_rows_f32<<<rp, 256, 0, stream_>>>(T.p, didx, rows, d_.dout, dout_p_, t_);
    k_gather_rows_f32<<<rp, 256, 0, stream_>>>(M.p, didx, rows, d_.dout, dout_p_, m_);
    forward(x_, rp, y_, true, stream_);
    const double loss = backward(t_, m_, rp, rows, stream_);
    return loss;
}

void LeafNet::train_host(const float* x, const float* t, const float* mask, int n, int epochs, int batch, float lr,
                         uint64_t seed, float* losses) {
    if (n <= 0 || epochs <= 0 || batch <= 0 || batch % 128) throw Error("invalid argument: training sizes");
    ensure_rows(batch);
    DevTable X(x, (size_t)n * d_.din), T(t, (size_t)n * d_.dout), M(mask, (size_t)n * d_.dout);
    DevBuf<int> idx_buf(batch);
    int* didx = idx_buf.p;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
    if (!s) s = 1;
    for (int ep = 0; ep < epochs; ep++) {
        for (int i = n - 1; i > 0; i--) std::swap(order[i], order[(size_t)(xs_next(s) % (uint64_t)(i + 1))]);
        double sum = 0.0;
        const int nb = std::max(1, n / batch);  // whole batches (one short batch when n < batch)
        for (int bi = 0; bi < nb; bi++) {
            const int b0 = bi * batch, rows = std::min(batch, n - b0);
            LCK(cudaMemcpyAsync(didx, order.data() + b0, rows * 4, cudaMemcpyHostToDevice, stream_));
            k_gather_rows_bf16<<<batch, 256, 0, stream_>>>(X.p, didx, rows, d_.din, din_p_, x_);
            k_gather_rows_f32<<<batch, 256, 0, stream_>>>(T.p, didx, rows, d_.dout, dout_p_, t_);
            k_gather_rows_f32<<<batch, 256, 0, stream_>>>(M.p, didx, rows, d_.dout, dout_p_, m_);
            forward(x_, batch, y_, true, stream_);
            sum += backward(t_, m_, batch, rows, stream_);
            adam(lr, ++adam_t_, stream_);
        }
        check(stream_);
        if (losses) losses[ep] = (float)(sum / std::max(nb, 1));
    }
}

// ---------------------------------------------------------------- leaves
namespace {
__device__ __forceinline__ float block_sum(float v, float* red) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();  // red may still be read from a previous call
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    float s = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];  // same order in every thread
    return s;
}
struct LeafDev {
    const LeafItem* leaves;
    const uint8_t* cards;
    int ncards;
    uint64_t board_mask;
    const float* reach[2];
    size_t rstr[2];
    const uint64_t* hmask[2];
    const uint16_t* combo[2];
    const int16_t* hand_of[2];
    int nh[2];
    __nv_bfloat16* x;
    int din_p;
    float* y;
    int dout_p;
    float* mass;
    float* err;
};
// one row per (leaf, turn card): the reach sums, then the input row
__global__ void k_leaf_gather(LeafDev L) {
    __shared__ float red[32];
    __shared__ float inv[2];
    const int row = blockIdx.x, li = row / L.ncards, c = L.cards[row % L.ncards];
    const LeafItem lf = L.leaves[li];
    for (int q = 0; q < 2; q++) {
        const float* r = L.reach[q] + (size_t)lf.rs[q] * L.rstr[q];
        float acc = 0.0f;
        for (int h = threadIdx.x; h < L.nh[q]; h += blockDim.x)
            if (!((L.hmask[q][h] >> c) & 1ull)) acc += r[h];
        const float m = block_sum(acc, red);
        if (threadIdx.x == 0) {
            L.mass[row * 2 + q] = m;
            inv[q] = m > 0.0f ? 1.0f / m : 0.0f;
        }
    }
    __syncthreads();
    const uint64_t onehot = L.board_mask | (1ull << c);
    __nv_bfloat16* xr = L.x + (size_t)row * L.din_p;
    for (int col = threadIdx.x; col < L.din_p; col += blockDim.x) {
        float v = 0.0f;
        if (col < 52) {
            v = ((onehot >> col) & 1ull) ? 1.0f : 0.0f;
        } else if (col == 52) {
            v = lf.pot / lf.stack;
        } else if (col < kLeafIn) {
            const int q = col < 53 + 1326 ? 0 : 1, cb = col - 53 - q * 1326;
            const int h = L.hand_of[q][cb];
            if (h >= 0 && !((L.hmask[q][h] >> c) & 1ull))
                v = L.reach[q][(size_t)lf.rs[q] * L.rstr[q] + h] * inv[q];
        }
        xr[col] = __float2bfloat16_rn(v);
    }
}
// per row: sum r0 y0 + sum r1 y1 over the combos (the zero-sum error)
__global__ void k_leaf_err(LeafDev L) {
    __shared__ float red[32];
    const int row = blockIdx.x;
    const __nv_bfloat16* xr = L.x + (size_t)row * L.din_p + 53;
    const float* yr = L.y + (size_t)row * L.dout_p;
    float acc = 0.0f;
    for (int k = threadIdx.x; k < kLeafOut; k += blockDim.x) acc += __bfloat162float(xr[k]) * yr[k];
    const float e = block_sum(acc, red);
    if (threadIdx.x == 0) L.err[row] = e;
}
// one block per leaf: player p's values, summed over the turn cards
__global__ void k_leaf_scatter(LeafDev L, int p, float* cfv, size_t stride) {
    const int li = blockIdx.x;
    const LeafItem lf = L.leaves[li];
    const float inv = 1.0f / 45.0f;
    for (int h = threadIdx.x; h < L.nh[p]; h += blockDim.x) {
        const uint64_t hm = L.hmask[p][h];
        const int cb = L.combo[p][h];
        float acc = 0.0f;
        for (int j = 0; j < L.ncards; j++) {
            const int c = L.cards[j];
            if ((hm >> c) & 1ull) continue;
            const int row = li * L.ncards + j;
            const float yv = L.y[(size_t)row * L.dout_p + p * 1326 + cb] - 0.5f * L.err[row];
            acc += yv * lf.pot * L.mass[row * 2 + (1 - p)];
        }
        cfv[(size_t)lf.cslot * stride + h] = acc * inv;
    }
}
template <class T>
T* dcopy(const T* h, size_t n) {
    T* p = dnew<T>(n);
    if (n) LCK(cudaMemcpy(p, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return p;
}
}  // namespace

LeafEvaluator::LeafEvaluator(std::shared_ptr<LeafNet> net, const Spot& sp, const std::vector<LeafItem>& leaves)
    : net_(std::move(net)) {
    if (!net_) throw Error("invalid argument: no leaf network");
    if (net_->dims().din != kLeafIn || net_->dims().dout != kLeafOut)
        throw Error("invalid argument: the leaf network must map " + std::to_string(kLeafIn) + " inputs to " +
                    std::to_string(kLeafOut) + " outputs");
    if (sp.board.size() != 3) throw Error("invalid argument: a depth-limited solve needs a flop spot");
    if (leaves.empty()) throw Error("invalid argument: the spot has no turn leaves");
    nleaves_ = (int)leaves.size();
    std::vector<uint8_t> cards;
    for (uint8_t b : sp.board) board_mask_ |= 1ull << b;
    for (int c = 0; c < 52; c++)
        if (!((board_mask_ >> c) & 1ull)) cards.push_back((uint8_t)c);
    ncards_ = (int)cards.size();
    rows_ = nleaves_ * ncards_;
    rows_p_ = pad128(rows_);
    for (int q = 0; q < 2; q++) {
        const Hands& H = sp.hands[q];
        nh_[q] = (int)H.size();
        std::vector<uint16_t> combo(H.size());
        std::vector<int16_t> hand_of(1326, -1);
        for (size_t h = 0; h < H.size(); h++) {
            const int hi = H.c1[h], lo = H.c2[h];
            combo[h] = (uint16_t)(hi * (hi - 1) / 2 + lo);
            hand_of[combo[h]] = (int16_t)h;
        }
        hmask_[q] = dcopy(H.mask.data(), H.mask.size());
        combo_[q] = dcopy(combo.data(), combo.size());
        hand_of_[q] = dcopy(hand_of.data(), hand_of.size());
    }
    leaves_ = dcopy(leaves.data(), leaves.size());
    cards_ = dcopy(cards.data(), cards.size());
    x_ = dnew<__nv_bfloat16>((size_t)rows_p_ * net_->din_pad());  // padding rows stay zero
    y_ = dnew<float>((size_t)rows_p_ * net_->dout_pad());
    mass_ = dnew<float>((size_t)rows_ * 2);
    err_ = dnew<float>((size_t)rows_);
    net_->reserve_rows(rows_p_);
}

LeafEvaluator::~LeafEvaluator() {
    for (void* p : {(void*)leaves_, (void*)cards_, (void*)hmask_[0], (void*)hmask_[1], (void*)combo_[0],
                    (void*)combo_[1], (void*)hand_of_[0], (void*)hand_of_[1], (void*)x_, (void*)y_, (void*)mass_,
                    (void*)err_})
        cudaFree(p);
}

void LeafEvaluator::run(int p, const float* reach0, size_t rstr0, const float* reach1, size_t rstr1, float* cfv,
                        size_t cfv_stride, cudaStream_t s) {
    LeafDev L;
    L.leaves = leaves_;
    L.cards = cards_;
    L.ncards = ncards_;
    L.board_mask = board_mask_;
    L.reach[0] = reach0;
    L.reach[1] = reach1;
    L.rstr[0] = rstr0;
    L.rstr[1] = rstr1;
    for (int q = 0; q < 2; q++) {
        L.hmask[q] = hmask_[q];
        L.combo[q] = combo_[q];
        L.hand_of[q] = hand_of_[q];
        L.nh[q] = nh_[q];
    }
    L.x = x_;
    L.din_p = net_->din_pad();
    L.y = y_;
    L.dout_p = net_->dout_pad();
    L.mass = mass_;
    L.err = err_;
    k_leaf_gather<<<rows_, 256, 0, s>>>(L);
    net_->forward_device(x_, rows_p_, y_, s);
    k_leaf_err<<<rows_, 256, 0, s>>>(L);
    k_leaf_scatter<<<nleaves_, 256, 0, s>>>(L, p, cfv, cfv_stride);
    LCK(cudaGetLastError());
}

}  // namespace gtob
