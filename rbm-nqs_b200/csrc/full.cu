// full.cu -- exact enumeration (full_sampler::sample, full_sampler.cpp:43-186)
// on the device: the state list in the reference's order, the weights
// p = |psi|^2 and the weighted aggregators (aggregator.cpp:190-239).
//
// Order: the low `bits` bits (sampler.full.n_parallel_bits) select a block
// b; within a block the high n - bits bits run through the Gray code, state
// k = b 2^(n-bits) + i being b | gray(i) << bits (full_sampler.cpp:63-136).
// The weights are |psi|^2 exp(-max_k 2 Re log psi_k): every aggregate is
// normalised by the total weight, so the common factor cancels, and no
// state overflows.  All sums run in a fixed order (deterministic).
#include <cstdint>

#include "sr.cuh"

namespace rbmnqs {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double bred_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double r = red[0];
    for (int i = 1; i < nw; i++) r += red[i];
    return r;
}
__device__ __forceinline__ double bred_max(double v, double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double r = red[0];
    for (int i = 1; i < nw; i++) r = fmax(r, red[i]);
    return r;
}

__global__ void full_states_kernel(uint32_t* samples, int n, int bits) {
    const int64_t N = int64_t(1) << n;
    const int hb = n - bits;
    const uint64_t lo = (uint64_t(1) << hb) - 1;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t b = (uint64_t)k >> hb, i = (uint64_t)k & lo;
        const uint64_t num = b | ((i ^ (i >> 1)) << bits);
        reinterpret_cast<uint4*>(samples)[k] = make_uint4((uint32_t)num, (uint32_t)(num >> 32), 0u, 0u);
    }
}

__global__ void full_max_partial(const double2* lp, int64_t N, double* part) {
    __shared__ double red[32];
    double m = -1.0e308;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, 2.0 * lp[k].x);
    m = bred_max(m, red);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}

// every block reduces the same maxima in the same order, so all agree on mx
__global__ void full_weight_partial(const double2* lp, int64_t N, double* p, double* part, FullStatsDev* fs) {
    __shared__ double red[32];
    double m = -1.0e308;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) m = fmax(m, part[i]);
    const double mx = bred_max(m, red);
    double w = 0, w2 = 0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) {
        const double pk = exp(2.0 * lp[k].x - mx);
        p[k] = pk;
        w += pk;
        w2 += pk * pk;
    }
    w = bred_sum(w, red);
    w2 = bred_sum(w2, red);
    if (threadIdx.x == 0) {
        part[gridDim.x + 2 * blockIdx.x] = w;
        part[gridDim.x + 2 * blockIdx.x + 1] = w2;
        if (blockIdx.x == 0) fs->mx = mx;
    }
}

__global__ void full_finalize(const double* part, int G, FullStatsDev* fs) {
    if (threadIdx.x == 0) {
        double W = 0, W2 = 0;
        for (int b = 0; b < G; b++) {
            W += part[G + 2 * b];
            W2 += part[G + 2 * b + 1];
        }
        fs->W = W;
        fs->W2 = W2;
        fs->vfac = W / (W - W2 / W);  // aggregator.cpp:150-157 (ptotal - wsum2 / ptotal)
    }
}

template <typename TO>
__global__ void full_center_kernel(TO* O, const double* p, const FullStatsDev* fs, const double2* d, int64_t N,
                                   int P) {
    const double scale = (double)N / fs->W;
    const int64_t total = N * (int64_t)P;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / P;
        const int q = (int)(i - k * P);
        const double s = sqrt(scale * p[k]);
        const TO o = O[i];
        const double2 dq = d[q];
        O[i].x = s * ((double)o.x - dq.x);
        O[i].y = s * ((double)o.y - dq.y);
    }
}

// aggregator::aggregate / finalize with weights (aggregator.cpp:190-239) for
// the energy: M2 = sum p |E - mu|^2; bins of N / n_bins consecutive states
// give M2b = sum_b W_b |mean_b - mu|^2 (the weighted Welford recurrences of
// the reference sum to these); variances divide by W - W2 / W.  A bin whose
// weights all underflow to zero contributes nothing.
__global__ void energy_stats_weighted_kernel(const double2* E, const double* p, int64_t N, int n_bins,
                                             const double2* emean, const FullStatsDev* fs, EpochStatsDev* out) {
    __shared__ double red[32];
    const double2 mu = *emean;
    double m2 = 0;
    int finite = 1;
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
        const double2 e = E[i];
        if (!isfinite(e.x) || !isfinite(e.y)) finite = 0;
        const double dx = e.x - mu.x, dy = e.y - mu.y;
        m2 += p[i] * (dx * dx + dy * dy);
    }
    m2 = bred_sum(m2, red);
    const int64_t bs = N / n_bins;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    double m2b = 0;
    for (int b = wid; b < n_bins; b += nwarp) {  // one warp per bin
        double wb = 0, sx = 0, sy = 0;
        for (int64_t i = (int64_t)b * bs + lane; i < (int64_t)(b + 1) * bs; i += 32) {
            const double pi = p[i];
            wb += pi;
            sx += pi * E[i].x;
            sy += pi * E[i].y;
        }
        for (int o = 16; o; o >>= 1) {
            wb += __shfl_xor_sync(0xffffffffu, wb, o);
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
        if (lane == 0 && wb > 0) {
            const double dx = sx / wb - mu.x, dy = sy / wb - mu.y;
            m2b += wb * (dx * dx + dy * dy);
        }
    }
    m2b = bred_sum(m2b, red);
    const double nf = bred_sum((double)finite, red);
    if (threadIdx.x == 0) {
        double tau = 0;
        if (n_bins > 1 && !(m2 == 0 && m2b == 0)) {
            const double r = (double)bs * m2b / m2;
            tau = 0.5 * ((r < 1 ? 1 : r) - 1);
        }
        const double den = fs->W - fs->W2 / fs->W;
        double v = m2 / den, vb = m2b / den;
        v = v < 0 ? 0 : v;
        vb = vb < 0 ? 0 : vb;
        out->energy = mu;
        out->var = v;
        out->var_binned = vb;
        out->tau = tau;
        out->stddev = n_bins > 1 ? sqrt(vb / n_bins) : sqrt(v / (double)N);
        out->acceptance = 0;
        out->finite = nf == (double)blockDim.x ? 1 : 0;
    }
}

__global__ void wmean_kernel(const double2* E, const double* p, int64_t N, const FullStatsDev* fs, double2* mu) {
    __shared__ double red[32];
    double sx = 0, sy = 0;
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
        sx += p[i] * E[i].x;
        sy += p[i] * E[i].y;
    }
    sx = bred_sum(sx, red);
    sy = bred_sum(sy, red);
    if (threadIdx.x == 0) *mu = make_double2(sx / fs->W, sy / fs->W);
}

__global__ void full_state_vector_kernel(const double2* lp, const uint32_t* samples, int64_t N,
                                         const FullStatsDev* fs, double2* psi) {
    const double half = 0.5 * fs->mx, inv = 1.0 / sqrt(fs->W);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += (int64_t)gridDim.x * blockDim.x) {
        const uint4 s = reinterpret_cast<const uint4*>(samples)[k];
        const uint64_t num = (uint64_t)s.x | ((uint64_t)s.y << 32);
        const double2 l = lp[k];
        const double a = exp(l.x - half) * inv;
        double sn, cs;
        sincos(l.y, &sn, &cs);
        psi[num] = make_double2(a * cs, a * sn);
    }
}

int grid_for(int64_t n) {
    const int64_t b = (n + kThreads - 1) / kThreads;
    return (int)(b < 4 * 148 ? (b < 1 ? 1 : b) : 4 * 148);
}

}  // namespace

cudaError_t launch_full_states(uint32_t* samples, int n, int bits, cudaStream_t st) {
    full_states_kernel<<<grid_for(int64_t(1) << n), kThreads, 0, st>>>(samples, n, bits);
    return cudaGetLastError();
}

cudaError_t launch_full_weights(const double2* logpsi, int64_t N, double* p, double* part, FullStatsDev* fs,
                                cudaStream_t st) {
    full_max_partial<<<kFullBlocks, kThreads, 0, st>>>(logpsi, N, part);
    full_weight_partial<<<kFullBlocks, kThreads, 0, st>>>(logpsi, N, p, part, fs);
    full_finalize<<<1, 32, 0, st>>>(part, kFullBlocks, fs);
    return cudaGetLastError();
}

cudaError_t launch_full_center(void* O, int fp64, const double* p, const FullStatsDev* fs, const double2* d,
                               int64_t N, int P, cudaStream_t st) {
    const int g = grid_for(N * (int64_t)P);
    if (fp64)
        full_center_kernel<double2><<<g, kThreads, 0, st>>>(static_cast<double2*>(O), p, fs, d, N, P);
    else
        full_center_kernel<float2><<<g, kThreads, 0, st>>>(static_cast<float2*>(O), p, fs, d, N, P);
    return cudaGetLastError();
}

cudaError_t launch_energy_stats_weighted(const double2* E, const double* p, int64_t N, int n_bins,
                                         const double2* emean, const FullStatsDev* fs, EpochStatsDev* out,
                                         cudaStream_t st) {
    energy_stats_weighted_kernel<<<1, 1024, 0, st>>>(E, p, N, n_bins, emean, fs, out);
    return cudaGetLastError();
}

cudaError_t launch_wmean(const double2* E, const double* p, int64_t N, const FullStatsDev* fs, double2* mu,
                         cudaStream_t st) {
    wmean_kernel<<<1, 1024, 0, st>>>(E, p, N, fs, mu);
    return cudaGetLastError();
}

cudaError_t launch_full_state_vector(const double2* logpsi, const uint32_t* samples, int64_t N,
                                     const FullStatsDev* fs, double2* psi, cudaStream_t st) {
    full_state_vector_kernel<<<grid_for(N), kThreads, 0, st>>>(logpsi, samples, N, fs, psi);
    return cudaGetLastError();
}

}  // namespace rbmnqs
