// The learned turn-leaf value network: a fully connected net (BF16 weights
// and activations, FP32 accumulation and master weights) whose every matrix
// product runs on one hand-written tcgen05 kernel -- operands staged by TMA
// in 128-byte-swizzled shared memory, the accumulator in tensor memory, bias,
// GELU and GELU' fused into the epilogue.  Forward, backward and Adam run on
// the device; inputs and targets come from the host (training) or from the
// engine's leaf gather (depth-limited solves).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "../host/plan.hpp"

namespace gtob {

// C[M x N] = A[M x K] * B[N x K]^T, both operands row-major bf16 with K
// contiguous; M, N multiples of 128, K a multiple of 64.  Epilogue per
// element, in order: + bias[col]; pre = v (f32); v *= gelu'(gmul[row, col]);
// v = gelu(v); out_f32 = v; out_bf16 = bf16(v).  Null pointers skip a step.
struct GemmEpilogue {
    const float* bias = nullptr;
    float* pre = nullptr;
    int ld_pre = 0;
    const float* gmul = nullptr;
    int ld_gmul = 0;
    bool gelu = false;
    float* out_f32 = nullptr;
    int ld_f32 = 0;
    __nv_bfloat16* out_bf16 = nullptr;
    int ld_bf16 = 0;
};
// err: device word; bit 4 is set when a wait inside the kernel gave up
void gemm_bf16_tn(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, int N, int K, const GemmEpilogue& e,
                  unsigned* err, cudaStream_t s);

// mean ms of reps products on m x k, n x k operands (f32 output), events
double gemm_time_ms(int m, int n, int k, int reps);

struct LeafNetDims {
    int din = 0, dh = 0, nhidden = 0, dout = 0;  // as given (unpadded)
};

class LeafNet {
  public:
    LeafNet(const LeafNetDims& d, uint64_t seed);
    ~LeafNet();
    const LeafNetDims& dims() const { return d_; }
    int layers() const { return d_.nhidden + 1; }
    // layer l's weights [out x in] and bias [out], unpadded, f32 (the masters)
    void get_params(int l, float* w, float* b) const;
    void set_params(int l, const float* w, const float* b);
    void get_grads(int l, float* w, float* b) const;
    // rows x din host inputs -> rows x dout host outputs
    void forward_host(const float* x, int rows, float* y);
    // one forward + backward over rows samples (masked mean squared error);
    // gradients stay on the device (get_grads); returns the loss
    double gradients_host(const float* x, const float* t, const float* mask, int rows);
    // epochs of Adam over n samples in shuffled batches; per-epoch mean loss
    void train_host(const float* x, const float* t, const float* mask, int n, int epochs, int batch, float lr,
                    uint64_t seed, float* losses);
    // device buffers for rows_pad rows: call before capturing forward_device
    void reserve_rows(int rows_pad) { ensure_rows(rows_pad); }
    // device-side forward over rows padded inputs (bf16, rows_pad x din_pad,
    // rows_pad a multiple of 128) into f32 outputs (rows_pad x dout_pad)
    void forward_device(const __nv_bfloat16* x, int rows_pad, float* y, cudaStream_t s);
    int din_pad() const { return din_p_; }
    int dout_pad() const { return dout_p_; }
    unsigned* err_word() const { return err_; }
    uint32_t kernel_launches() const { return launches_; }

  private:
    struct Layer;
    void ensure_rows(int rows_pad);
    void forward(const __nv_bfloat16* x, int rows_pad, float* y, bool keep, cudaStream_t s);
    double backward(const float* t, const float* mask, int rows_pad, int rows, cudaStream_t s);
    void adam(float lr, int step, cudaStream_t s);
    void check(cudaStream_t s);
    LeafNetDims d_;
    int din_p_ = 0, dh_p_ = 0, dout_p_ = 0;
    std::vector<std::unique_ptr<Layer>> L_;
    int rows_cap_ = 0;
    __nv_bfloat16 *x_ = nullptr, *xt_ = nullptr, *dyb_ = nullptr, *dyt_ = nullptr;
    float *y_ = nullptr, *dy_ = nullptr, *t_ = nullptr, *m_ = nullptr;
    double* loss_ = nullptr;
    unsigned* err_ = nullptr;
    int adam_t_ = 0;
    uint32_t launches_ = 0;
    cudaStream_t stream_ = nullptr;
};

// The turn-leaf inputs and outputs of a depth-limited flop plan.  Inputs per
// (leaf, turn card c) row, kLeafIn = 2705 values: the board and c one-hot
// (52), pot / remaining stack, and each player's reach at the leaf over the
// 1326 combos (hands holding c or absent are 0) divided by its sum.  Outputs
// per row, kLeafOut = 2652: each player's counterfactual values over the
// combos, divided by pot x the opponent's reach sum.  A leaf's values for p
// are those of every turn card, zero-sum corrected (the outputs shifted by
// half of sum r0 y0 + sum r1 y1), scaled back and added over the cards a hand
// does not hold, times 1/45 (the chance node's 1 / (46 - street)).
constexpr int kLeafIn = 52 + 1 + 2 * 1326;
constexpr int kLeafOut = 2 * 1326;

class LeafEvaluator {
  public:
    LeafEvaluator(std::shared_ptr<LeafNet> net, const Spot& spot, const std::vector<LeafItem>& leaves);
    ~LeafEvaluator();
    // the leaves' values for player p into cfv (slot stride cfv_stride)
    void run(int p, const float* reach0, size_t rstr0, const float* reach1, size_t rstr1, float* cfv,
             size_t cfv_stride, cudaStream_t s);
    int rows() const { return rows_; }
    uint32_t launches_per_run() const { return 3 + (uint32_t)net_->layers(); }
    LeafNet& net() { return *net_; }

  private:
    std::shared_ptr<LeafNet> net_;
    int nleaves_ = 0, ncards_ = 0, rows_ = 0, rows_p_ = 0;
    int nh_[2] = {0, 0};
    uint64_t board_mask_ = 0;
    LeafItem* leaves_ = nullptr;
    uint8_t* cards_ = nullptr;            // the turn cards, ascending
    uint64_t* hmask_[2] = {nullptr, nullptr};
    uint16_t* combo_[2] = {nullptr, nullptr};  // hand -> combo
    int16_t* hand_of_[2] = {nullptr, nullptr}; // combo -> hand (-1: none)
    __nv_bfloat16* x_ = nullptr;
    float* y_ = nullptr;
    float* mass_ = nullptr;  // [row][2]
    float* err_ = nullptr;   // [row]
};

}  // namespace gtob
