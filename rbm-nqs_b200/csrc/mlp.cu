// mlp.cu -- proposal-network kernels: one tcgen05 BF16 GEMM with fused
// epilogues (bias + GELU, GELU backward, FP32 split-K partials) and the
// elementwise / transpose / reduction / Adam kernels around it.
//
// GEMM: C[M x N] = A[M x K] B[N x K]^T, both operands K-major BF16 in
// global memory, N <= 256 and K a multiple of 64.  One CTA (128 threads)
// computes one 128-row tile over one K range of up to 256 (four 64-wide
// chunks): TMA (128-byte swizzle) brings the whole A and B tiles in at once,
// one thread issues K/16 tcgen05.mma kind::f16 into a TMEM accumulator of N
// columns, and four warps read it back (tcgen05.ld) for the epilogue.  Every
// wait is bounded (error flag, no hang).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "mlp.cuh"
#include "sr.cuh"
#include "tc_common.cuh"

namespace rbmnqs {
namespace {

using namespace tc;

constexpr int kRows = 128;       // M tile
constexpr int kChunk = 64;       // K elements per 128-byte swizzle row
constexpr int kMaxChunks = 4;    // K per CTA <= 256
constexpr int kMaxN = 256;

enum EpiMode : int { kStoreF32 = 0, kBiasGelu = 1, kBiasF32 = 2, kGeluBwd = 3 };

struct Epi {
    int mode;
    int stall;             // test fault 2: the copies are not issued, the bounded wait runs out
    float* f32;            // kStoreF32: [nsplit][Mtot][ld]; kBiasGelu: Z; kBiasF32: logits
    __nv_bfloat16* bf;     // kBiasGelu: activation; kGeluBwd: gradient
    const float* bias;     // kBiasGelu, kBiasF32
    const float* z;        // kGeluBwd: pre-activation Z [Mtot][ld]
    int ld;                // leading dimension of every output (= N)
    int mtot;              // rows of the output
};

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float z) {
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B (format 1),
// both K-major, M = 128, N as given.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// grid (M / 128, nsplit, output tiles); K range of this CTA: [blockIdx.y *
// nchunks * 64, +nchunks * 64); output columns [blockIdx.z * N, +N) (N is
// the tile width, at most 128 when the output is split).  Eight warps: warp
// w reads TMEM lanes 32 (w mod 4) .. +31 and the 16-column chunks of parity
// w / 4 in the epilogue.
__global__ void __launch_bounds__(256, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int N,
                     int nchunks, Epi epi, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar, done_bar;
    __shared__ uint32_t tmem_base;
    __shared__ int ok_load;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const uint32_t a_base = base, b_base = base + nchunks * (kRows * 128);
    const int m0 = blockIdx.x * kRows, k0 = blockIdx.y * nchunks * kChunk, n0 = blockIdx.z * N;
    const uint32_t ncols = N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));

    if (tid == 0) {
        mbar_init(smem_u32(&full_bar), 1);
        mbar_init(smem_u32(&done_bar), 1);
        ok_load = 1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    if (tid == 0) {
        const uint32_t fb = smem_u32(&full_bar);
        if (!epi.stall) {
            mbar_expect_tx(fb, (uint32_t)nchunks * (kRows * 128 + N * 128));
            for (int c = 0; c < nchunks; c++) {
                tma_load_2d(a_base + c * (kRows * 128), &mapA, fb, k0 + c * kChunk, m0);
                tma_load_2d(b_base + c * (N * 128), &mapB, fb, k0 + c * kChunk, n0);
            }
        }
        // under the test fault no copy is in flight and nothing arrives:
        // the wait gives up after a short limit
        if (epi.stall ? mbar_wait_n(fb, 0, 4096u) : mbar_wait(fb, 0)) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t id = idesc_bf16(N);
            for (int c = 0; c < nchunks; c++)
#pragma unroll
                for (int k = 0; k < kChunk / 16; k++) {
                    const uint64_t da = desc_sw128(a_base + c * (kRows * 128) + k * 32);
                    const uint64_t db = desc_sw128(b_base + c * (N * 128) + k * 32);
                    mma_bf16(tmem, da, db, id, (c > 0 || k > 0) ? 1u : 0u);
                }
            mma_commit(smem_u32(&done_bar));
        } else {
            ok_load = 0;
            atomicExch(err, 1);
            if (!epi.stall) (void)mbar_wait(fb, 0);  // drain the copies (bounded)
        }
    }
    __syncthreads();
    int done = 1;
    if (ok_load) done = (int)mbar_wait(smem_u32(&done_bar), 0);
    const bool have = __syncthreads_and(done) && ok_load;
    if (!have && tid == 0 && ok_load) atomicExch(err, 2);
    asm volatile("tcgen05.fence::after_thread_sync;");

    const int quarter = warp & 3;
    const int row = m0 + 32 * quarter + lane;
    __syncwarp();
    for (int cl = 16 * (warp >> 2); cl < N; cl += 32) {
        uint32_t r[16];
        __syncwarp();
        if (have) {
            tmem_ld16(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)cl, r);
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) r[j] = 0u;
        }
        if (row >= epi.mtot) continue;
        const int c0 = n0 + cl;  // output column
        const size_t o = (size_t)row * epi.ld + c0;
        if (epi.mode == kStoreF32) {
            float* dst = epi.f32 + (size_t)blockIdx.y * epi.mtot * epi.ld + o;
#pragma unroll
            for (int j = 0; j < 16; j += 4)
                *reinterpret_cast<float4*>(dst + j) = make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]),
                                                                  __uint_as_float(r[j + 2]), __uint_as_float(r[j + 3]));
        } else if (epi.mode == kBiasGelu) {
            __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const float z = __uint_as_float(r[j]) + epi.bias[c0 + j];
                epi.f32[o + j] = z;
                hb[j] = __float2bfloat16_rn(gelu_f(z));
            }
            *reinterpret_cast<uint4*>(epi.bf + o) = *reinterpret_cast<const uint4*>(hb);
            *reinterpret_cast<uint4*>(epi.bf + o + 8) = *reinterpret_cast<const uint4*>(hb + 8);
        } else if (epi.mode == kBiasF32) {
#pragma unroll
            for (int j = 0; j < 16; j++) epi.f32[o + j] = __uint_as_float(r[j]) + epi.bias[c0 + j];
        } else {  // kGeluBwd
            __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
            for (int j = 0; j < 16; j++) hb[j] = __float2bfloat16_rn(__uint_as_float(r[j]) * gelu_grad_f(epi.z[o + j]));
            *reinterpret_cast<uint4*>(epi.bf + o) = *reinterpret_cast<const uint4*>(hb);
            *reinterpret_cast<uint4*>(epi.bf + o + 8) = *reinterpret_cast<const uint4*>(hb + 8);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
    }
}

// configurations (bits; set = spin down) -> +-1 BF16 rows [rows][cols], rows
// >= B and columns >= n zero
__global__ void encode_spins(const uint32_t* __restrict__ bits, int B, int n, int rows, int cols,
                             __nv_bfloat16* __restrict__ X) {
    const size_t total = (size_t)rows * cols;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / cols), c = (int)(i % cols);
        float v = 0.f;
        if (b < B && c < n) v = ((bits[4 * b + (c >> 5)] >> (c & 31)) & 1u) ? -1.f : 1.f;
        X[i] = __float2bfloat16_rn(v);
    }
}

// dL/dlogits = (sigmoid(l) - t) / B (BF16) and per-block loss partials
__global__ void bce_grad(const float* __restrict__ L, const uint32_t* __restrict__ tbits, int B, int n, int rows,
                         int cols, __nv_bfloat16* __restrict__ G, float* __restrict__ lossp) {
    __shared__ float red[32];
    const size_t total = (size_t)rows * cols;
    float acc = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / cols), c = (int)(i % cols);
        float g = 0.f;
        if (b < B && c < n) {
            const float l = L[i];
            const float t = (float)((tbits[4 * b + (c >> 5)] >> (c & 31)) & 1u);
            g = (1.f / (1.f + expf(-l)) - t) / (float)B;
            acc += (fmaxf(l, 0.f) + log1pf(expf(-fabsf(l))) - t * l) / (float)B;  // softplus(l) - t l
        }
        G[i] = __float2bfloat16_rn(g);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
        lossp[blockIdx.x] = s;
    }
}

// Soft-target softmax cross entropy, one warp per row: with p = softmax(l)
// over the n logical outputs, dL/dl = (p - t) / B and the loss is
// -(1/B) sum_m t_m log p_m; targets tg[b][n] (rows sum to 1).  Padded rows
// and columns get zero gradient.
__global__ void softmax_ce_grad(const float* __restrict__ L, const float* __restrict__ tg, int B, int n, int rows,
                                int cols, __nv_bfloat16* __restrict__ G, float* __restrict__ lossp) {
    __shared__ float red[32];
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    float acc = 0.f;
    for (int b = blockIdx.x * wpb + (threadIdx.x >> 5); b < rows; b += gridDim.x * wpb) {
        const float* lr = L + (size_t)b * cols;
        __nv_bfloat16* gr = G + (size_t)b * cols;
        if (b >= B) {
            for (int c = lane; c < cols; c += 32) gr[c] = __float2bfloat16_rn(0.f);
            continue;
        }
        float mx = -INFINITY;
        for (int c = lane; c < n; c += 32) mx = fmaxf(mx, lr[c]);
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        float se = 0.f;
        for (int c = lane; c < n; c += 32) se += expf(lr[c] - mx);
        for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
        const float lse = mx + logf(se);
        for (int c = lane; c < cols; c += 32) {
            float g = 0.f;
            if (c < n) {
                const float lp = lr[c] - lse, t = tg[(size_t)b * n + c];
                g = (expf(lp) - t) / (float)B;
                acc -= t * lp / (float)B;
            }
            gr[c] = __float2bfloat16_rn(g);
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < wpb; w++) s += red[w];
        lossp[blockIdx.x] = s;
    }
}

__global__ void sum_loss(const float* lossp, int n, float* out) {
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int i = 0; i < n; i++) s += lossp[i];
        *out = s;
    }
}

// [R][C] -> [C][ldo] BF16 (first R columns) through 32 x 32 shared tiles
__global__ void transpose_bf16(const __nv_bfloat16* __restrict__ in, int R, int C, __nv_bfloat16* __restrict__ out,
                               int ldo) {
    __shared__ __nv_bfloat16 t[32][34];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int r = ty; r < 32; r += 8)
        if (r0 + r < R && c0 + tx < C) t[r][tx] = in[(size_t)(r0 + r) * C + c0 + tx];
    __syncthreads();
    for (int c = ty; c < 32; c += 8)
        if (c0 + c < C && r0 + tx < R) out[(size_t)(c0 + c) * ldo + r0 + tx] = t[tx][c];
}

// gradient of a layer: dW = sum over splits (FP32), db = column sums of G
// dW = the sum of the split-K partials (blocks [0, wblocks), grid-stride);
// db = the column sums of G over the rows (blocks from wblocks on, 32
// columns each: the block's warps take interleaved rows with four
// accumulators, then the warp partials are added in warp order)
__global__ void __launch_bounds__(256) finish_grads(const float* __restrict__ part, int nsplit, int out, int in,
                                                    const __nv_bfloat16* __restrict__ G, int rows,
                                                    float* __restrict__ dW, float* __restrict__ db, int wblocks) {
    if ((int)blockIdx.x < wblocks) {
        const size_t total = (size_t)out * in;
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)wblocks * blockDim.x) {
            float s = 0.f;
            for (int k = 0; k < nsplit; k++) s += part[(size_t)k * total + i];
            dW[i] = s;
        }
        return;
    }
    __shared__ float red[8][33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int c = (blockIdx.x - wblocks) * 32 + lane;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    if (c < out) {
        int b = w;
        for (; b + 3 * nw < rows; b += 4 * nw) {
            a0 += __bfloat162float(G[(size_t)b * out + c]);
            a1 += __bfloat162float(G[(size_t)(b + nw) * out + c]);
            a2 += __bfloat162float(G[(size_t)(b + 2 * nw) * out + c]);
            a3 += __bfloat162float(G[(size_t)(b + 3 * nw) * out + c]);
        }
        for (; b < rows; b += nw) a0 += __bfloat162float(G[(size_t)b * out + c]);
    }
    red[w][lane] = (a0 + a1) + (a2 + a3);
    __syncthreads();
    if (w == 0 && c < out) {
        float t = red[0][lane];
        for (int j = 1; j < nw; j++) t += red[j][lane];
        db[c] = t;
    }
}

// Adam on the flat FP32 master parameters
__global__ void adam_step(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                          const float* __restrict__ g, size_t n, float lr, float bc1, float bc2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = 0.9f * m[i] + 0.1f * gi;
        const float vi = 0.999f * v[i] + 0.001f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
    }
}

// BF16 copy [out][in] and transposed copy [in][out] of one FP32 weight
__global__ void to_bf16(const float* __restrict__ W, int out, int in, __nv_bfloat16* __restrict__ Wb,
                        __nv_bfloat16* __restrict__ Wt) {
    const size_t total = (size_t)out * in;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const __nv_bfloat16 h = __float2bfloat16_rn(W[i]);
        Wb[i] = h;
        if (Wt) Wt[(i % in) * out + i / in] = h;
    }
}

__global__ void init_normal(float* w, size_t n, float std, uint64_t seed, uint32_t stream) {
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint4 r = philox4x32(make_uint4((uint32_t)i, (uint32_t)(i >> 32), stream, 7), key);
        // Box-Muller on two 24-bit uniforms in (0, 1]
        const float u1 = ((r.x >> 8) + 1) * (1.0f / 16777216.0f), u2 = (r.y >> 8) * (1.0f / 16777216.0f);
        w[i] = std * sqrtf(-2.f * logf(u1)) * cospif(2.f * u2);
    }
}

// rows of a B operand's TMA box for an output of N columns: 128-column
// output tiles when N is a larger multiple of 128
static int b_tile(int N) { return (N > 128 && N % 128 == 0) ? 128 : N; }

cudaError_t encode_map(void* dst, const void* base, int rows, int cols, int box_rows) {
    auto fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kChunk, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(reinterpret_cast<CUtensorMap*>(dst), CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                          const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int grid_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }

}  // namespace

// ---------------------------------------------------------------------------
static cudaError_t gemm(const void* mapA, const void* mapB, int M, int N, int K, int nsplit, const Epi& e0, int* err,
                        cudaStream_t st) {
    Epi e = e0;
    e.stall = test_fault() == 2 ? 1 : 0;
    // M multiple of 128, N multiple of 16 (<= 256), K = nsplit * nchunks * 64;
    // outputs wider than 128 columns (multiples of 128) in 128-column tiles
    // (the B map's box is b_tile(N) rows)
    const int nchunks = K / (kChunk * nsplit);
    if (M % kRows || N % 16 || N > kMaxN || nchunks < 1 || nchunks > kMaxChunks || nchunks * kChunk * nsplit != K)
        return cudaErrorInvalidValue;
    const int NT = b_tile(N);
    const int smem = nchunks * (kRows * 128 + NT * 128) + 1024;
    cudaError_t r = ensure_dynamic_smem(reinterpret_cast<const void*>(gemm_bf16_kernel), smem);
    if (r != cudaSuccess) return r;
    gemm_bf16_kernel<<<dim3(M / kRows, nsplit, N / NT), 256, smem, st>>>(
        *reinterpret_cast<const CUtensorMap*>(mapA), *reinterpret_cast<const CUtensorMap*>(mapB), NT, nchunks, e, err);
    return cudaGetLastError();
}

Mlp::Mlp(const MlpDims& d, int max_batch, cudaStream_t st) : d_(d), st_(st) {
    d_.in_p = (d.n_in + 63) / 64 * 64;
    d_.out_p = (d.n_out + 63) / 64 * 64;
    bmax_ = (max_batch + 255) / 256 * 256;
    auto al = [&](auto*& p, size_t n) {
        void* q = nullptr;
        if (cudaMalloc(&q, n) != cudaSuccess) throw cudaErrorMemoryAllocation;
        cudaMemsetAsync(q, 0, n, st_);
        allocs_.push_back(q);
        p = reinterpret_cast<std::remove_reference_t<decltype(p)>>(q);
    };
    const size_t np = n_params();
    al(master_, np * 4);
    al(m_, np * 4);
    al(v_, np * 4);
    al(grad_, np * 4);
    const int I = d_.in_p, H1 = d_.h1, H2 = d_.h2, Oo = d_.out_p, Bm = bmax_;
    al(W1_, (size_t)H1 * I * 2);
    al(W2_, (size_t)H2 * H1 * 2);
    al(W3_, (size_t)Oo * H2 * 2);
    al(W2t_, (size_t)H1 * H2 * 2);
    al(W3t_, (size_t)H2 * Oo * 2);
    al(X0_, (size_t)Bm * I * 2);
    al(A1_, (size_t)Bm * H1 * 2);
    al(A2_, (size_t)Bm * H2 * 2);
    al(G1_, (size_t)Bm * H1 * 2);
    al(G2_, (size_t)Bm * H2 * 2);
    al(G3_, (size_t)Bm * Oo * 2);
    al(X0t_, (size_t)Bm * I * 2);
    al(A1t_, (size_t)Bm * H1 * 2);
    al(A2t_, (size_t)Bm * H2 * 2);
    // gradient transposes: rows padded to the 128-row tile of the
    // weight-gradient GEMM (the padding rows stay zero)
    auto r128 = [](int r) { return (r + kRows - 1) / kRows * kRows; };
    al(G1t_, (size_t)Bm * r128(H1) * 2);
    al(G2t_, (size_t)Bm * r128(H2) * 2);
    al(G3t_, (size_t)Bm * r128(Oo) * 2);
    al(Z1_, (size_t)Bm * H1 * 4);
    al(Z2_, (size_t)Bm * H2 * 4);
    al(L_, (size_t)Bm * Oo * 4);
    const int maxsplit = Bm / 256;
    size_t pmax = std::max({(size_t)H1 * I, (size_t)H2 * H1, (size_t)Oo * H2});
    al(part_, (size_t)maxsplit * pmax * 4);
    al(lossp_, 148 * 8 * 4);
    al(err_, 16);
    // tensor maps: forward A operands (box 128 rows) / B operands (box = N rows)
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t x) {
        if (x != cudaSuccess && e == cudaSuccess) e = x;
    };
    chk(encode_map(mX0_.m, X0_, Bm, I, kRows));
    chk(encode_map(mA1_.m, A1_, Bm, H1, kRows));
    chk(encode_map(mA2_.m, A2_, Bm, H2, kRows));
    chk(encode_map(mG3_.m, G3_, Bm, Oo, kRows));
    chk(encode_map(mG2_.m, G2_, Bm, H2, kRows));
    chk(encode_map(mW1_.m, W1_, H1, I, b_tile(H1)));
    chk(encode_map(mW2_.m, W2_, H2, H1, b_tile(H2)));
    chk(encode_map(mW3_.m, W3_, Oo, H2, b_tile(Oo)));
    chk(encode_map(mW3t_.m, W3t_, H2, Oo, b_tile(H2)));
    chk(encode_map(mW2t_.m, W2t_, H1, H2, b_tile(H1)));
    // weight-gradient GEMMs: A = G^T [out][B] (128-row tiles), B = X^T [in][B] (box = in rows)
    chk(encode_map(mG3t_.m, G3t_, r128(Oo), Bm, kRows));
    chk(encode_map(mG2t_.m, G2t_, r128(H2), Bm, kRows));
    chk(encode_map(mG1t_.m, G1t_, r128(H1), Bm, kRows));
    chk(encode_map(mA2t_.m, A2t_, H2, Bm, b_tile(H2)));
    chk(encode_map(mA1t_.m, A1t_, H1, Bm, b_tile(H1)));
    chk(encode_map(mX0t_.m, X0t_, I, Bm, b_tile(I)));
    if (e != cudaSuccess) throw e;
}

Mlp::~Mlp() {
    for (void* p : allocs_) cudaFree(p);
}

size_t Mlp::off_W(int l) const {
    const size_t w1 = (size_t)d_.h1 * d_.in_p, w2 = (size_t)d_.h2 * d_.h1;
    return l == 0 ? 0 : (l == 1 ? w1 + d_.h1 : w1 + d_.h1 + w2 + d_.h2);
}
size_t Mlp::off_b(int l) const {
    const int rows[3] = {d_.h1, d_.h2, d_.out_p};
    const int cols[3] = {d_.in_p, d_.h1, d_.h2};
    return off_W(l) + (size_t)rows[l] * cols[l];
}
size_t Mlp::n_params() const { return off_b(2) + d_.out_p; }

cudaError_t Mlp::refresh_bf16(cudaStream_t st) {
    to_bf16<<<grid_for((size_t)d_.h1 * d_.in_p), 256, 0, st>>>(master_ + off_W(0), d_.h1, d_.in_p, W1_, nullptr);
    to_bf16<<<grid_for((size_t)d_.h2 * d_.h1), 256, 0, st>>>(master_ + off_W(1), d_.h2, d_.h1, W2_, W2t_);
    to_bf16<<<grid_for((size_t)d_.out_p * d_.h2), 256, 0, st>>>(master_ + off_W(2), d_.out_p, d_.h2, W3_, W3t_);
    return cudaGetLastError();
}

// logical [W1 (h1 x n_in), b1, W2, b2, W3 (n_out x h2), b3] <-> padded master
cudaError_t Mlp::set_params(const float* host) {
    std::vector<float> pad(n_params(), 0.f);
    const int rows[3] = {d_.h1, d_.h2, d_.n_out}, cols[3] = {d_.n_in, d_.h1, d_.h2};
    const int pcols[3] = {d_.in_p, d_.h1, d_.h2};
    size_t src = 0;
    for (int l = 0; l < 3; l++) {
        for (int r = 0; r < rows[l]; r++)
            for (int c = 0; c < cols[l]; c++) pad[off_W(l) + (size_t)r * pcols[l] + c] = host[src++];
        for (int r = 0; r < rows[l]; r++) pad[off_b(l) + r] = host[src++];
    }
    cudaError_t e = cudaMemcpyAsync(master_, pad.data(), pad.size() * 4, cudaMemcpyHostToDevice, st_);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st_);  // pad is a stack temporary
    if (e != cudaSuccess) return e;
    cudaMemsetAsync(m_, 0, n_params() * 4, st_);
    cudaMemsetAsync(v_, 0, n_params() * 4, st_);
    step_ = 0;
    return refresh_bf16(st_);
}

cudaError_t Mlp::get_params(float* host) {
    std::vector<float> pad(n_params());
    cudaError_t e = cudaMemcpyAsync(pad.data(), master_, pad.size() * 4, cudaMemcpyDeviceToHost, st_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
    if (e != cudaSuccess) return e;
    const int rows[3] = {d_.h1, d_.h2, d_.n_out}, cols[3] = {d_.n_in, d_.h1, d_.h2};
    const int pcols[3] = {d_.in_p, d_.h1, d_.h2};
    size_t dst = 0;
    for (int l = 0; l < 3; l++) {
        for (int r = 0; r < rows[l]; r++)
            for (int c = 0; c < cols[l]; c++) host[dst++] = pad[off_W(l) + (size_t)r * pcols[l] + c];
        for (int r = 0; r < rows[l]; r++) host[dst++] = pad[off_b(l) + r];
    }
    return cudaSuccess;
}

cudaError_t Mlp::init_random(float std, uint64_t seed) {
    cudaMemsetAsync(master_, 0, n_params() * 4, st_);
    const int rows[3] = {d_.h1, d_.h2, d_.n_out}, pcols[3] = {d_.in_p, d_.h1, d_.h2};
    for (int l = 0; l < 3; l++) {
        // logical block rows x pcols (padding columns of W1 are multiplied by
        // zero inputs; padding rows of W3 only produce ignored logits)
        const size_t n = (size_t)rows[l] * pcols[l];
        init_normal<<<grid_for(n), 256, 0, st_>>>(master_ + off_W(l), n, std, seed, (uint32_t)l);
    }
    cudaMemsetAsync(m_, 0, n_params() * 4, st_);
    cudaMemsetAsync(v_, 0, n_params() * 4, st_);
    step_ = 0;
    return refresh_bf16(st_);
}

cudaError_t Mlp::forward(const uint32_t* spins, int B, cudaStream_t st) {
    if (B < 1 || B > bmax_) return cudaErrorInvalidValue;
    const int M = (B + 255) / 256 * 256;  // the same padded rows as train_step
    const int I = d_.in_p, H1 = d_.h1, H2 = d_.h2, Oo = d_.out_p;
    encode_spins<<<grid_for((size_t)M * I), 256, 0, st>>>(spins, B, d_.n_in, M, I, X0_);
    Epi e{};
    e.mode = kBiasGelu;
    e.ld = H1;
    e.mtot = M;
    e.f32 = Z1_;
    e.bf = A1_;
    e.bias = master_ + off_b(0);
    cudaError_t r = gemm(mX0_.m, mW1_.m, M, H1, I, 1, e, err_, st);
    if (r != cudaSuccess) return r;
    e.ld = H2;
    e.f32 = Z2_;
    e.bf = A2_;
    e.bias = master_ + off_b(1);
    if ((r = gemm(mA1_.m, mW2_.m, M, H2, H1, 1, e, err_, st)) != cudaSuccess) return r;
    e.mode = kBiasF32;
    e.ld = Oo;
    e.f32 = L_;
    e.bf = nullptr;
    e.bias = master_ + off_b(2);
    return gemm(mA2_.m, mW3_.m, M, Oo, H2, 1, e, err_, st);
}

cudaError_t Mlp::train_step(const uint32_t* spins, const uint32_t* targets, int B, float lr, cudaStream_t st,
                            float* loss_dev, bool apply) {
    cudaError_t r = forward(spins, B, st);
    if (r != cudaSuccess) return r;
    const int M = (B + 255) / 256 * 256;  // split-K chunks of 256 samples
    if (M > bmax_) return cudaErrorInvalidValue;
    const int nb = grid_for((size_t)M * d_.out_p);
    bce_grad<<<nb, 256, 0, st>>>(L_, targets, B, d_.n_out, M, d_.out_p, G3_, lossp_);
    if (loss_dev) sum_loss<<<1, 32, 0, st>>>(lossp_, nb, loss_dev);
    return backward_step(B, lr, st, apply);
}

cudaError_t Mlp::train_step_soft(const uint32_t* spins, const float* targets, int B, float lr, cudaStream_t st,
                                 float* loss_dev, bool apply) {
    cudaError_t r = forward(spins, B, st);
    if (r != cudaSuccess) return r;
    const int M = (B + 255) / 256 * 256;
    if (M > bmax_) return cudaErrorInvalidValue;
    const int nb = std::min(148 * 4, (M + 7) / 8);
    softmax_ce_grad<<<nb, 256, 0, st>>>(L_, targets, B, d_.n_out, M, d_.out_p, G3_, lossp_);
    if (loss_dev) sum_loss<<<1, 32, 0, st>>>(lossp_, nb, loss_dev);
    return backward_step(B, lr, st, apply);
}

cudaError_t Mlp::backward_step(int B, float lr, cudaStream_t st, bool apply) {
    cudaError_t r;
    const int M = (B + 255) / 256 * 256;
    const int I = d_.in_p, H1 = d_.h1, H2 = d_.h2, Oo = d_.out_p;
    // dA2 = G3 W3 -> G2 = dA2 * gelu'(Z2); dA1 = G2 W2 -> G1
    Epi e{};
    e.mode = kGeluBwd;
    e.mtot = M;
    e.ld = H2;
    e.bf = G2_;
    e.z = Z2_;
    if ((r = gemm(mG3_.m, mW3t_.m, M, H2, Oo, 1, e, err_, st)) != cudaSuccess) return r;
    e.ld = H1;
    e.bf = G1_;
    e.z = Z1_;
    if ((r = gemm(mG2_.m, mW2t_.m, M, H1, H2, 1, e, err_, st)) != cudaSuccess) return r;
    // transposed operands for the weight gradients (K = samples)
    auto tr = [&](const __nv_bfloat16* in, int C, __nv_bfloat16* out) {
        transpose_bf16<<<dim3((C + 31) / 32, M / 32), 256, 0, st>>>(in, M, C, out, bmax_);
    };
    tr(X0_, I, X0t_);
    tr(A1_, H1, A1t_);
    tr(A2_, H2, A2t_);
    tr(G1_, H1, G1t_);
    tr(G2_, H2, G2t_);
    tr(G3_, Oo, G3t_);
    const int ns = M / 256;
    Epi p{};
    p.mode = kStoreF32;
    p.f32 = part_;
    // dW3 = G3^T A2 [Oo x H2], dW2 = G2^T A1 [H2 x H1], dW1 = G1^T X0 [H1 x I]
    struct L {
        const void *a, *b;
        int out, in;
        const __nv_bfloat16* G;
        int layer;
    } ls[3] = {{mG3t_.m, mA2t_.m, Oo, H2, G3_, 2}, {mG2t_.m, mA1t_.m, H2, H1, G2_, 1}, {mG1t_.m, mX0t_.m, H1, I, G1_, 0}};
    for (auto& l : ls) {
        p.ld = l.in;
        p.mtot = l.out;
        const int mrows = (l.out + kRows - 1) / kRows * kRows;
        if ((r = gemm(l.a, l.b, mrows, l.in, M, ns, p, err_, st)) != cudaSuccess) return r;
        const int wb = grid_for((size_t)l.out * l.in), cb = (l.out + 31) / 32;
        finish_grads<<<wb + cb, 256, 0, st>>>(part_, ns, l.out, l.in, l.G, M, grad_ + off_W(l.layer),
                                              grad_ + off_b(l.layer), wb);
    }
    if (!apply) return cudaGetLastError();
    step_++;
    const float bc1 = 1.f - powf(0.9f, (float)step_), bc2 = 1.f - powf(0.999f, (float)step_);
    adam_step<<<grid_for(n_params()), 256, 0, st>>>(master_, m_, v_, grad_, n_params(), lr, bc1, bc2);
    return refresh_bf16(st);
}

cudaError_t Mlp::intermediate(int which, int B, float* host, int* cols) {
    const int H1 = d_.h1, H2 = d_.h2, Oo = d_.out_p;
    const void* src = nullptr;
    int c = 0;
    bool bf = true;
    switch (which) {
        case 0: src = A1_, c = H1; break;
        case 1: src = A2_, c = H2; break;
        case 2: src = Z1_, c = H1, bf = false; break;
        case 3: src = Z2_, c = H2, bf = false; break;
        case 4: src = G1_, c = H1; break;
        case 5: src = G2_, c = H2; break;
        case 6: src = G3_, c = Oo; break;
        default: return cudaErrorInvalidValue;
    }
    if (cols) *cols = c;
    if (!host) return cudaSuccess;
    const size_t n = (size_t)B * c;
    cudaError_t e;
    if (bf) {
        std::vector<__nv_bfloat16> t(n);
        e = cudaMemcpyAsync(t.data(), src, n * 2, cudaMemcpyDeviceToHost, st_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
        for (size_t i = 0; i < n; i++) host[i] = __bfloat162float(t[i]);
    } else {
        e = cudaMemcpyAsync(host, src, n * 4, cudaMemcpyDeviceToHost, st_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
    }
    return e;
}

int Mlp::error_flag_host() {
    int h = 0;
    cudaMemcpy(&h, err_, sizeof(int), cudaMemcpyDeviceToHost);
    return h;
}

}  // namespace rbmnqs
