// mlp.cuh -- the proposal network (learned multi-spin Metropolis proposals):
// 3-layer MLP n_in -> h1 -> h2 -> n_out with GELU, BF16 weights and
// activations, FP32 accumulation, forward and backward on tcgen05 tensor
// cores, Adam on FP32 master weights.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace rbmnqs {

struct MlpDims {
    int n_in = 128, h1 = 256, h2 = 256, n_out = 128;  // logical sizes
    int in_p = 128, out_p = 128;                      // padded to multiples of 64
};

// Device-side network state and work buffers for batches up to max_batch.
class Mlp {
   public:
    Mlp(const MlpDims& d, int max_batch, cudaStream_t st);
    ~Mlp();
    Mlp(const Mlp&) = delete;
    Mlp& operator=(const Mlp&) = delete;

    const MlpDims& dims() const { return d_; }
    int max_batch() const { return bmax_; }
    size_t n_params() const;
    // flat parameters [W1 (h1 x n_in), b1, W2 (h2 x h1), b2, W3 (n_out x h2), b3], row-major [out][in]
    cudaError_t set_params(const float* host);
    cudaError_t get_params(float* host);
    // N(0, std) weights, zero biases (Philox, seeded)
    cudaError_t init_random(float std, uint64_t seed);

    // logits [B][out_p] (FP32, device) of configurations spins[B][4] (device)
    cudaError_t forward(const uint32_t* spins, int B, cudaStream_t st);
    const float* logits() const { return L_; }
    // One Adam step on the BCE loss of logits against flip masks targets[B][4]
    // (device): loss -> *loss_dev (FP32, device scalar) when non-null.
    cudaError_t train_step(const uint32_t* spins, const uint32_t* targets, int B, float lr, cudaStream_t st,
                           float* loss_dev, bool apply);
    // The same step on the soft-target softmax cross entropy
    // -(1/B) sum_b sum_m t[b][m] log softmax(logits[b])_m, targets[B][n_out]
    // (FP32, device, rows summing to 1).
    cudaError_t train_step_soft(const uint32_t* spins, const float* targets, int B, float lr, cudaStream_t st,
                                float* loss_dev, bool apply);
    // gradient buffers (FP32, device) in the flat parameter layout, valid after train_step
    const float* grads() const { return grad_; }
    // intermediate tensors for tests: which = 0 a1, 1 a2, 2 z1, 3 z2, 4 g1, 5 g2, 6 g3 (rows x cols as float)
    cudaError_t intermediate(int which, int B, float* host, int* cols);
    int error_flag_host();
    // device address of the pipeline error flag, and its reset
    const int* error_flag() const { return err_; }
    cudaError_t clear_error(cudaStream_t st) { return cudaMemsetAsync(err_, 0, sizeof(int), st); }

   private:
    MlpDims d_;
    int bmax_;
    cudaStream_t st_;
    // FP32 master parameters, Adam moments, gradients (flat layout, padded sizes)
    float *master_ = nullptr, *m_ = nullptr, *v_ = nullptr, *grad_ = nullptr;
    int step_ = 0;
    // BF16 weights [out][in] and transposes [in][out] (padded)
    __nv_bfloat16 *W1_ = nullptr, *W2_ = nullptr, *W3_ = nullptr, *W2t_ = nullptr, *W3t_ = nullptr;
    // activations [bmax][.] and their transposes [.][bmax]
    __nv_bfloat16 *X0_ = nullptr, *A1_ = nullptr, *A2_ = nullptr, *G1_ = nullptr, *G2_ = nullptr, *G3_ = nullptr;
    __nv_bfloat16 *X0t_ = nullptr, *A1t_ = nullptr, *A2t_ = nullptr, *G1t_ = nullptr, *G2t_ = nullptr, *G3t_ = nullptr;
    float *Z1_ = nullptr, *Z2_ = nullptr, *L_ = nullptr, *part_ = nullptr, *lossp_ = nullptr;
    int* err_ = nullptr;
    // tensor maps (CUtensorMap, 128 B each)
    struct Map {
        alignas(64) unsigned char m[128];
    };
    Map mX0_, mA1_, mA2_, mW1_, mW2_, mW3_, mG2_, mG3_, mW2t_, mW3t_;
    Map mG1t_, mG2t_, mG3t_, mX0t_, mA1t_, mA2t_;
    std::vector<void*> allocs_;
    size_t off_W(int l) const;
    size_t off_b(int l) const;
    cudaError_t refresh_bf16(cudaStream_t st);
    // backward from dL/dlogits in G3 (after a forward of B rows), gradients,
    // and the Adam step when apply
    cudaError_t backward_step(int B, float lr, cudaStream_t st, bool apply);
};

}  // namespace rbmnqs
