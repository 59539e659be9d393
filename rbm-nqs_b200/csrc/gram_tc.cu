// gram_tc.cu -- the SR Gram S = <conj(O - d) (O - d)^T> on the 5th-generation
// tensor cores (tcgen05, kind::f16, accumulator in TMEM).
//
// Real embedding: with X[n][2p] = Re(O - d)[n][p], X[n][2p+1] = Im(...), the
// real Gram G = X^T X gives S_pq = (G[2p][2q] + G[2p+1][2q+1]
//                                   + i (G[2p][2q+1] - G[2p+1][2q])) / N.
// Split precision in FP16: every real row r of X is scaled by a power of two
// s_r (max_n |X[n][r]| s_r in [2^13, 2^14), from a row-maximum pass, so that
// no value overflows FP16 and, since max <= sqrt(N) rms, typical values stay
// far from the FP16 subnormals); X s = Xh + Xl with Xh = fp16(X s), Xl =
// fp16(X s - Xh).  G s_r s_c ~= Xh Xh^T + Xh Xl^T + Xl Xh^T accumulated in
// FP32 inside TMEM (the dropped Xl Xl^T term is ~2^-22 relative: the same
// 11 + 11 significant bits as a TF32 hi / lo split, at twice the tensor rate
// and half the bytes); split-K partial tiles are summed in FP64 and the
// scales divided out.
//
// Layout: Xh, Xl are K-major [R][K] fp16 (row r = real parameter 2p or
// 2p+1, K = samples, both zero-padded to tile multiples).  One CTA owns one
// 128x128 tile (tp <= tq) of G and one range of K: TMA (128-byte swizzle,
// box 64 x 128) fills a three-stage ring of {Ah, Al, Bh, Bl} tiles; one thread
// issues three tcgen05.mma (M = N = 128, K = 16) per k-step, four k-steps per
// stage, and commits each stage back to its "empty" barrier; four warps read
// the accumulator with tcgen05.ld and store the FP32 partial tile.  Every
// wait is bounded: on timeout the kernel records an error code, stops
// issuing, drains and frees its TMEM.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <utility>
#include <vector>
#include <cstdint>

#include "common.cuh"
#include "gram_tc.cuh"
#include "tc_common.cuh"

namespace rbmnqs {
namespace {

using namespace tc;

constexpr int TILE = 128;                     // M = N tile (rows of G)
constexpr int BK = 64;                        // K per stage (128 B of fp16)
constexpr int STAGE_TILE_BYTES = TILE * BK * 2;  // 16 KB
constexpr int STAGE_BYTES = 4 * STAGE_TILE_BYTES;  // Ah, Al, Bh, Bl
constexpr int STAGES = 3;
constexpr long kMaxPartialBytes = 256L << 20;  // split-K partial tiles
constexpr int kMaxAccumKb = 128;               // preferred longest FP32 accumulation per CTA (8192 samples)

// kind::f16 instruction descriptor: FP32 accumulate, FP16 A and B (format
// 0), both K-major, N = 128, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(TILE >> 3) << 17) |
                            ((uint32_t)(TILE >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// power-of-two scale of a real row from its maximum |value|: max s in
// [2^13, 2^14) (1 for an all-zero row)
__device__ __forceinline__ float row_scale(float mx) {
    if (!(mx > 0.f)) return 1.f;
    int e;
    frexpf(mx, &e);  // mx = f 2^e, f in [0.5, 1)
    return ldexpf(1.f, 14 - e);
}

__global__ void __launch_bounds__(128, 1)
    gram_tc_kernel(const __grid_constant__ CUtensorMap mh, const __grid_constant__ CUtensorMap ml, int ntile,
                   int nkb_total, float* __restrict__ part, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], done_bar;
    __shared__ uint32_t tmem_base;
    __shared__ int failed, mma_count;

    // tile (tp <= tq) of the upper triangle and this CTA's k-block range
    int t = blockIdx.x, tp = 0;
    while (t >= ntile - tp) {
        t -= ntile - tp;
        tp++;
    }
    const int tq = tp + t;
    const int split = blockIdx.y, nsplit = gridDim.y;
    const int kb0 = (int)((long)nkb_total * split / nsplit), kb1 = (int)((long)nkb_total * (split + 1) / nsplit);
    const int nkb = kb1 - kb0;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;  // 1024-B aligned ring

    if (tid == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(smem_u32(&full_bar[s]), 1);
            mbar_init(smem_u32(&empty_bar[s]), 1);
        }
        mbar_init(smem_u32(&done_bar), 1);
        failed = 0;
        mma_count = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(TILE));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    if (tid == 0 && nkb > 0) {
        auto stage_addr = [&](int s, int which) { return base + s * STAGE_BYTES + which * STAGE_TILE_BYTES; };
        auto load = [&](int i) {  // k-block i of this CTA into stage i % STAGES
            const int s = i % STAGES;
            const uint32_t fb = smem_u32(&full_bar[s]);
            const int x = (kb0 + i) * BK;
            mbar_expect_tx(fb, STAGE_BYTES);
            tma_load_2d(stage_addr(s, 0), &mh, fb, x, tp * TILE);
            tma_load_2d(stage_addr(s, 1), &ml, fb, x, tp * TILE);
            tma_load_2d(stage_addr(s, 2), &mh, fb, x, tq * TILE);
            tma_load_2d(stage_addr(s, 3), &ml, fb, x, tq * TILE);
        };
        bool ok = true;
        int issued = 0, consumed = 0;  // loads issued, k-blocks whose MMAs were issued
        for (; issued < nkb && issued < STAGES; issued++) load(issued);
        for (int i = 0; i < nkb; i++) {
            const int s = i % STAGES;
            if (!(ok = mbar_wait(smem_u32(&full_bar[s]), (i / STAGES) & 1))) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int k = 0; k < BK / 16; k++) {
                const uint32_t off = k * 32;  // 16 fp16 = 32 B along K inside the swizzled row
                const uint64_t ah = desc_sw128(stage_addr(s, 0) + off), al = desc_sw128(stage_addr(s, 1) + off);
                const uint64_t bh = desc_sw128(stage_addr(s, 2) + off), bl = desc_sw128(stage_addr(s, 3) + off);
                mma_f16(tmem, ah, bh, (i > 0 || k > 0) ? 1u : 0u);
                mma_f16(tmem, ah, bl, 1u);
                mma_f16(tmem, al, bh, 1u);
            }
            mma_commit(smem_u32(&empty_bar[s]));
            consumed = i + 1;
            // refill the stage of k-block i-1 once its MMAs are done (those
            // of k-block i stay queued meanwhile)
            if (i >= 1 && issued < nkb) {
                const int j = i - 1;
                if (!(ok = mbar_wait(smem_u32(&empty_bar[j % STAGES]), (j / STAGES) & 1))) break;
                load(issued++);
            }
        }
        if (consumed > 0) mma_commit(smem_u32(&done_bar));
        if (!ok) {
            failed = 1;
            atomicExch(err, 1);
            // drain (bounded): loads in flight that no MMA consumed
            for (int i = consumed; i < issued; i++) (void)mbar_wait(smem_u32(&full_bar[i % STAGES]), (i / STAGES) & 1);
        }
        mma_count = consumed;
    }
    __syncthreads();
    // all MMAs retired (also after a failure); 'have' is block-uniform so the
    // warp-collective TMEM loads below run converged
    const int done = mma_count > 0 ? (int)mbar_wait(smem_u32(&done_bar), 0) : 1;
    const bool have = __syncthreads_and(done) && nkb > 0 && !failed;
    if (!have && tid == 0 && !failed && nkb > 0) atomicExch(err, 2);
    asm volatile("tcgen05.fence::after_thread_sync;");
    // epilogue: warp w reads TMEM lanes (rows) 32w..32w+31, 16 columns at a time
    const int row = 32 * warp + lane;
    float* dst = part + (((size_t)split * gridDim.x + blockIdx.x) * TILE + row) * TILE;
    __syncwarp();
    for (int c = 0; c < TILE; c += 16) {
        uint32_t r[16];
        if (have) {
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c, r);
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) r[j] = 0u;
        }
#pragma unroll
        for (int j = 0; j < 16; j += 4)
            *reinterpret_cast<float4*>(dst + c + j) =
                make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]), __uint_as_float(r[j + 2]),
                            __uint_as_float(r[j + 3]));
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TILE));
    }
}

// Row maxima: rmax[2p] = max_n |Re(O - d)[n][p]|, rmax[2p+1] the same for
// Im (rmax zeroed before; non-negative floats compare as their bit patterns).
template <typename TO>
__global__ void gram_rowmax(const TO* __restrict__ O, const double2* __restrict__ d, int N, int P,
                            unsigned int* __restrict__ rmax) {
    const int p = blockIdx.x * 32 + (threadIdx.x & 31);
    if (p >= P) return;
    const double2 dd = d[p];
    float mr = 0.f, mi = 0.f;
    auto take = [&](TO o) {
        float vr, vi;
        if constexpr (sizeof(TO) == 8) {
            vr = (float)((double)o.x - dd.x);
            vi = (float)((double)o.y - dd.y);
        } else {
            vr = (float)(o.x - dd.x);
            vi = (float)(o.y - dd.y);
        }
        mr = fmaxf(mr, fabsf(vr));
        mi = fmaxf(mi, fabsf(vi));
    };
    // four rows' loads in flight before their maxima (order-free)
    const int step = gridDim.y * (blockDim.x >> 5);
    int n = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (; n + 3 * step < N; n += 4 * step) {
        TO o[4];
#pragma unroll
        for (int u = 0; u < 4; u++) o[u] = O[(size_t)(n + u * step) * P + p];
#pragma unroll
        for (int u = 0; u < 4; u++) take(o[u]);
    }
    for (; n < N; n += step) take(O[(size_t)n * P + p]);
    atomicMax(rmax + 2 * p, __float_as_uint(mr));
    atomicMax(rmax + 2 * p + 1, __float_as_uint(mi));
}

// O (N x P complex, fp32 or fp64), d, row maxima -> K-major FP16 hi / lo
// planes Xh[r][n], Xl[r][n] of the scaled rows, r = 2p (real) / 2p+1 (imag);
// 32 x 32 transpose tiles through shared memory.
template <typename TO>
__global__ void gram_prep(const TO* __restrict__ O, const double2* __restrict__ d, const float* __restrict__ rmax,
                          int N, int P, int ld, __half* __restrict__ Xh, __half* __restrict__ Xl) {
    __shared__ float2 tile[32][33];
    const int n0 = blockIdx.x * 32, p0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const int n = n0 + r, p = p0 + tx;
        float2 v = make_float2(0.f, 0.f);
        if (n < N && p < P) {
            const double2 dd = d[p];
            if constexpr (sizeof(TO) == 8) {
                const float2 o = reinterpret_cast<const float2*>(O)[(size_t)n * P + p];
                v = make_float2((float)((double)o.x - dd.x), (float)((double)o.y - dd.y));
            } else {
                const double2 o = reinterpret_cast<const double2*>(O)[(size_t)n * P + p];
                v = make_float2((float)(o.x - dd.x), (float)(o.y - dd.y));
            }
        }
        tile[r][tx] = v;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int p = p0 + r, n = n0 + tx;
        if (p >= P || n >= N) continue;
        const float2 v = tile[tx][r];
        const float c[2] = {v.x, v.y};
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const float x = c[q] * row_scale(rmax[2 * p + q]);
            const __half h = __float2half_rn(x);
            Xh[(size_t)(2 * p + q) * ld + n] = h;
            Xl[(size_t)(2 * p + q) * ld + n] = __float2half_rn(x - __half2float(h));
        }
    }
}

// S[p][q] (p <= q) from the split partial tiles of G, the row scales divided
// out; Hermitian mirror.
__global__ void gram_tc_finalize(const float* __restrict__ part, const float* __restrict__ rmax, int ntile,
                                 int nsplit, int N, int P, double2* __restrict__ S) {
    const int nup = ntile * (ntile + 1) / 2;
    const size_t total = (size_t)P * P;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int p = (int)(i / P), q = (int)(i % P);
        if (q < p) continue;
        const int rr = 2 * p, cc = 2 * q;
        const int tp = rr / TILE, tq = cc / TILE;
        const int tile = tp * ntile - tp * (tp - 1) / 2 + (tq - tp);
        const int lr = rr % TILE, lc = cc % TILE;
        double g00 = 0, g11 = 0, g01 = 0, g10 = 0;
        for (int s = 0; s < nsplit; s++) {
            const float* T = part + ((size_t)s * nup + tile) * TILE * TILE;
            g00 += T[lr * TILE + lc];
            g11 += T[(lr + 1) * TILE + lc + 1];
            g01 += T[lr * TILE + lc + 1];
            g10 += T[(lr + 1) * TILE + lc];
        }
        const double sr0 = row_scale(rmax[rr]), sr1 = row_scale(rmax[rr + 1]);
        const double sc0 = row_scale(rmax[cc]), sc1 = row_scale(rmax[cc + 1]);
        g00 /= sr0 * sc0;
        g11 /= sr1 * sc1;
        g01 /= sr0 * sc1;
        g10 /= sr1 * sc0;
        double2 v = make_double2((g00 + g11) / N, (g01 - g10) / N);
        if (p == q) v.y = 0;
        S[i] = v;
        S[(size_t)q * P + p] = make_double2(v.x, -v.y);
    }
}

}  // namespace

size_t GramTC::partial_bytes() const { return (size_t)max_splits * (ntile * (ntile + 1) / 2) * TILE * TILE * 4; }

// Modelled time of a split count: CTAs run in waves of one per SM (the
// shared-memory ring takes most of an SM), each CTA streams its k-blocks and
// pays a fixed set-up and epilogue of about kOverheadKb k-blocks.
static double gram_cost(int nup, int nkb, int ns, int sms) {
    constexpr double kOverheadKb = 8.0;
    const long ctas = (long)nup * ns;
    const long waves = (ctas + sms - 1) / sms;
    return (double)waves * ((double)((nkb + ns - 1) / ns) + kOverheadKb);
}

int gram_tc_split_candidates(const GramTC& g, int* out, int max_out) {
    // the split counts within the partial-buffer bound, ordered by modelled cost
    const int nup = g.ntile * (g.ntile + 1) / 2, nkb = g.K / BK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    std::vector<std::pair<double, int>> c;
    for (int ns = 1; ns <= g.max_splits; ns++) c.push_back({gram_cost(nup, nkb, ns, sms), ns});
    std::stable_sort(c.begin(), c.end());
    int n = 0;
    for (const auto& e : c) {
        if (n >= max_out) break;
        out[n++] = e.second;
    }
    return n;
}

cudaError_t gram_tc_set_splits(GramTC* g, int ns) {
    if (ns < 1 || ns > g->max_splits) return cudaErrorInvalidValue;
    g->nsplit = ns;
    return cudaSuccess;
}

cudaError_t gram_tc_plan(int N, int P, GramTC* g) {
    g->N = N;
    g->P = P;
    g->R = ((2 * P + TILE - 1) / TILE) * TILE;
    g->K = ((N + BK - 1) / BK) * BK;
    g->ntile = g->R / TILE;
    const int nup = g->ntile * (g->ntile + 1) / 2;
    const int nkb = g->K / BK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // split counts: at most one k-block per split and partial tiles within
    // kMaxPartialBytes (splits are summed in FP64).  The default is the
    // lowest modelled cost (gram_cost) among the counts whose FP32
    // accumulation runs are at most kMaxAccumKb k-blocks, or the largest
    // allowed count when none is that short; rbmnqs_autotune_sr times the
    // cheapest candidates on the device.
    long cap = kMaxPartialBytes / ((long)nup * TILE * TILE * 4);
    if (cap < 1) cap = 1;
    if (cap > nkb) cap = nkb;
    g->max_splits = (int)cap;
    const int ns_min = std::min((int)cap, std::max(1, (nkb + kMaxAccumKb - 1) / kMaxAccumKb));
    int best = ns_min;
    double best_cost = gram_cost(nup, nkb, ns_min, sms);
    for (int ns = ns_min + 1; ns <= cap; ns++) {
        const double c = gram_cost(nup, nkb, ns, sms);
        if (c < best_cost) {
            best_cost = c;
            best = ns;
        }
    }
    g->nsplit = best;
    return cudaSuccess;
}

cudaError_t gram_tc_maps(GramTC* g, void* buf) {
    auto fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    const size_t pe = g->plane_elems();
    g->Xh = reinterpret_cast<__half*>(buf);
    g->Xl = g->Xh + pe;
    g->rmax = reinterpret_cast<float*>(g->Xl + pe);
    __half* Xh = g->Xh;
    __half* Xl = g->Xl;
    for (int which = 0; which < 2; which++) {
        CUtensorMap* m = reinterpret_cast<CUtensorMap*>(which == 0 ? g->map_h : g->map_l);
        const cuuint64_t dims[2] = {(cuuint64_t)g->K, (cuuint64_t)g->R};
        const cuuint64_t strides[1] = {(cuuint64_t)g->K * 2};
        const cuuint32_t box[2] = {BK, TILE};
        const cuuint32_t estr[2] = {1, 1};
        CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, which == 0 ? (void*)Xh : (void*)Xl, dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
    return cudaSuccess;
}

cudaError_t launch_gram_tc(const GramTC& g, const void* O, int fp64, const double2* d, float* part, int* err,
                           double2* S, cudaStream_t st) {
    cudaError_t e0 = cudaMemsetAsync(g.rmax, 0, (size_t)g.R * sizeof(float), st);
    if (e0 != cudaSuccess) return e0;
    unsigned int* rmu = reinterpret_cast<unsigned int*>(g.rmax);
    const dim3 mg((g.P + 31) / 32, std::max(1, std::min(64, (g.N + 255) / 256)));
    dim3 pg((g.N + 31) / 32, (g.P + 31) / 32);
    if (fp64) {
        gram_rowmax<double2><<<mg, 256, 0, st>>>((const double2*)O, d, g.N, g.P, rmu);
        gram_prep<double2><<<pg, 256, 0, st>>>((const double2*)O, d, g.rmax, g.N, g.P, g.K, g.Xh, g.Xl);
    } else {
        gram_rowmax<float2><<<mg, 256, 0, st>>>((const float2*)O, d, g.N, g.P, rmu);
        gram_prep<float2><<<pg, 256, 0, st>>>((const float2*)O, d, g.rmax, g.N, g.P, g.K, g.Xh, g.Xl);
    }
    const int smem = STAGES * STAGE_BYTES + 1024;
    cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(gram_tc_kernel), smem);
    if (e != cudaSuccess) return e;
    const int nup = g.ntile * (g.ntile + 1) / 2;
    const CUtensorMap* mh = reinterpret_cast<const CUtensorMap*>(g.map_h);
    const CUtensorMap* ml = reinterpret_cast<const CUtensorMap*>(g.map_l);
    gram_tc_kernel<<<dim3(nup, g.nsplit), 128, smem, st>>>(*mh, *ml, g.ntile, g.K / BK, part, err);
    gram_tc_finalize<<<296, 256, 0, st>>>(part, g.rmax, g.ntile, g.nsplit, g.N, g.P, S);
    return cudaGetLastError();
}

}  // namespace rbmnqs
