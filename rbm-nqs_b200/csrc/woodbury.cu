// woodbury.cu -- the direct SR solver (optimizer/direct_solver.cpp:31-59)
// for parameter counts whose P x P matrix S is not formed.
//
// The direct solver's system is S_reg x = F with
//   S_reg = S + Lambda,   S = (1/N) Abar^H Abar,   Abar = O - 1 d^T (N x P),
//   Lambda_p = S_pp (r1 (+ rd on non-neural p)) + r2 max(diag)
// (the diagonal scaled by 1 + r1 (+ rd) plus r2 max|diag|).  Lambda is
// diagonal and positive, so S_reg is Hermitian positive definite and its
// solution unique; with fewer samples than parameters it comes from the
// N x N system of the Woodbury identity:
//   x = Lambda^-1 F - Lambda^-1 Abar^H K^-1 Abar Lambda^-1 F,
//   K = N I + Abar Lambda^-1 Abar^H
// (N is the normalisation `norm`; d must be the mean of O's rows, as the
// aggregator's d is, for S = O^H O / N - conj(d) d^T = Abar^H Abar / N).
// K is formed by an FP64 Gram of the samples (64 x 64 tiles), factored by
// the cooperative blocked Cholesky of direct.cu, and the two products with
// Abar are one pass over O each.  FP64 throughout (O itself FP32 or FP64).
#include <algorithm>

#include "common.cuh"
#include "sr.cuh"

namespace rbmnqs {
namespace {

constexpr int kThreads = 256;
constexpr int kT = 64;   // K tile (rows n, columns m)
constexpr int kPc = 16;  // parameters per shared-memory chunk

__device__ __forceinline__ double2 oval(const float2* O, size_t i, double2 d) {
    const float2 v = O[i];
    return make_double2((double)v.x - d.x, (double)v.y - d.y);
}
__device__ __forceinline__ double2 oval(const double2* O, size_t i, double2 d) {
    const double2 v = O[i];
    return make_double2(v.x - d.x, v.y - d.y);
}

// S_pp = sum_n |Abar_np|^2 / norm: one thread per parameter, rows in order
template <typename TO>
__global__ void wb_spp(const TO* __restrict__ O, const double2* __restrict__ d, int N, int P, double norm,
                       double* __restrict__ spp) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const double2 dp = d[p];
        double s = 0;
        for (int n = 0; n < N; n++) {
            const double2 a = oval(O, (size_t)n * P + p, dp);
            s = fma(a.x, a.x, fma(a.y, a.y, s));
        }
        spp[p] = s / norm;
    }
}

// winv_p = 1 / Lambda_p, y = F / Lambda (spp: S_pp; max_diag: the maximum
// of the variance diagonal that sets the r2 shift)
__global__ void wb_scale(const double* __restrict__ spp, const double* max_diag, const ScheduleDev* sch, double r1_,
                         double r2_, double rd_, int P, int n_neural, const double2* __restrict__ F,
                         double* __restrict__ winv, double2* __restrict__ y) {
    const double r1 = sch ? sch->value[1] : r1_, r2 = sch ? sch->value[2] : r2_, rd = sch ? sch->value[3] : rd_;
    const double mx = *max_diag;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const double lam = spp[p] * (p < n_neural ? r1 : r1 + rd) + r2 * mx;
        const double w = 1.0 / lam;
        winv[p] = w;
        y[p] = make_double2(F[p].x * w, F[p].y * w);
    }
}

// u_n = sum_p Abar_np y_p: one warp per row, lanes over the parameters
template <typename TO>
__global__ void wb_rows(const TO* __restrict__ O, const double2* __restrict__ d, const double2* __restrict__ y, int N,
                        int P, double2* __restrict__ u) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; n < N; n += nw) {
        double ax = 0, ay = 0;
        for (int p = lane; p < P; p += 32) {
            const double2 a = oval(O, (size_t)n * P + p, d[p]), b = y[p];
            ax = fma(a.x, b.x, fma(-a.y, b.y, ax));
            ay = fma(a.x, b.y, fma(a.y, b.x, ay));
        }
        ax = warp_sum(ax);
        ay = warp_sum(ay);
        if (lane == 0) u[n] = make_double2(ax, ay);
    }
}

// K_nm = norm delta_nm + sum_p Abar_np winv_p conj(Abar_mp) for the tile pairs
// n0 <= m0 (blockIdx.x enumerates them), mirrored to the lower triangle.
// 16 x 16 threads, each a 4 x 4 block of outputs (rows ty + 16 i, columns
// tx + 16 j of the tile).
template <typename TO>
__global__ void __launch_bounds__(kThreads) wb_gram(const TO* __restrict__ O, const double2* __restrict__ d,
                                                    const double* __restrict__ winv, int N, int P, int ntile,
                                                    double norm, double2* __restrict__ K) {
    __shared__ double2 A[kT][kPc + 1], B[kT][kPc + 1];
    int t = blockIdx.x, bt = 0;
    while (t >= ntile - bt) {
        t -= ntile - bt;
        bt++;
    }
    const int n0 = bt * kT, m0 = (bt + t) * kT;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0, 0);
    for (int p0 = 0; p0 < P; p0 += kPc) {
        // A: rows n0.. weighted by winv; B: rows m0.. (conjugated at use)
        for (int e = threadIdx.x; e < kT * kPc; e += kThreads) {
            const int r = e / kPc, c = e % kPc, p = p0 + c;
            double2 a = make_double2(0, 0), b = make_double2(0, 0);
            if (p < P) {
                const double2 dp = d[p];
                if (n0 + r < N) {
                    a = oval(O, (size_t)(n0 + r) * P + p, dp);
                    const double w = winv[p];
                    a = make_double2(a.x * w, a.y * w);
                }
                if (m0 + r < N) b = oval(O, (size_t)(m0 + r) * P + p, dp);
            }
            A[r][c] = a;
            B[r][c] = b;
        }
        __syncthreads();
#pragma unroll 4
        for (int c = 0; c < kPc; c++) {
            double2 a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = A[ty + 16 * i][c];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = B[tx + 16 * j][c];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {  // a conj(b)
                    acc[i][j].x = fma(a[i].x, b[j].x, fma(a[i].y, b[j].y, acc[i][j].x));
                    acc[i][j].y = fma(a[i].y, b[j].x, fma(-a[i].x, b[j].y, acc[i][j].y));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int n = n0 + ty + 16 * i, m = m0 + tx + 16 * j;
            if (n >= N || m >= N || m < n) continue;
            double2 v = acc[i][j];
            if (n == m) v = make_double2(v.x + norm, 0.0);
            K[(size_t)n * N + m] = v;
            if (m != n) K[(size_t)m * N + n] = make_double2(v.x, -v.y);
        }
}

// x_p = y_p - winv_p sum_n conj(Abar_np) z_n: one thread per parameter, the
// rows streamed in order (coalesced across the parameters)
template <typename TO>
__global__ void wb_cols(const TO* __restrict__ O, const double2* __restrict__ d, const double2* __restrict__ z,
                        const double* __restrict__ winv, const double2* __restrict__ y, int N, int P,
                        double2* __restrict__ x) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const double2 dp = d[p];
        double sx = 0, sy = 0;
        for (int n = 0; n < N; n++) {
            const double2 a = oval(O, (size_t)n * P + p, dp), b = z[n];
            sx = fma(a.x, b.x, fma(a.y, b.y, sx));  // conj(a) b
            sy = fma(a.x, b.y, fma(-a.y, b.x, sy));
        }
        const double w = winv[p];
        x[p] = make_double2(y[p].x - w * sx, y[p].y - w * sy);
    }
}

}  // namespace

size_t woodbury_work_bytes(int N, int P) {
    return (size_t)P * (8 + 8 + 16) + (size_t)N * 16 * 3 + (size_t)N * N * 16 + sizeof(MfreeSync) + 1024;
}

WoodburyWork woodbury_carve(void* base, int N, int P) {
    WoodburyWork w{};
    auto* z = reinterpret_cast<double2*>(base);
    w.K = z;
    w.y = w.K + (size_t)N * N;
    w.u = w.y + P;
    w.z = w.u + N;
    w.work = w.z + N;
    w.winv = reinterpret_cast<double*>(w.work + N);
    w.spp = w.winv + P;
    w.sync = reinterpret_cast<MfreeSync*>(reinterpret_cast<uintptr_t>(w.spp + P) + 255 & ~uintptr_t(255));
    return w;
}

cudaError_t launch_woodbury_solve(const void* O, int fp64, const double2* d, int N, int P, int n_neural,
                                  double norm, const double2* F, double2* x, const double* max_diag,
                                  const ScheduleDev* sch, double r1, double r2, double rd, const WoodburyWork& w,
                                  CgResultDev* res, cudaStream_t st) {
    const int gp = std::max(1, std::min(148 * 8, (P + kThreads - 1) / kThreads));
    if (fp64)
        wb_spp<double2><<<gp, kThreads, 0, st>>>((const double2*)O, d, N, P, norm, w.spp);
    else
        wb_spp<float2><<<gp, kThreads, 0, st>>>((const float2*)O, d, N, P, norm, w.spp);
    wb_scale<<<gp, kThreads, 0, st>>>(w.spp, max_diag, sch, r1, r2, rd, P, n_neural, F, w.winv, w.y);
    const int ntile = (N + kT - 1) / kT;
    const int gr = std::max(1, std::min(148 * 8, (N + 7) / 8));
    if (fp64) {
        wb_rows<double2><<<gr, kThreads, 0, st>>>((const double2*)O, d, w.y, N, P, w.u);
        wb_gram<double2><<<ntile * (ntile + 1) / 2, kThreads, 0, st>>>((const double2*)O, d, w.winv, N, P, ntile,
                                                                        norm, w.K);
    } else {
        wb_rows<float2><<<gr, kThreads, 0, st>>>((const float2*)O, d, w.y, N, P, w.u);
        wb_gram<float2><<<ntile * (ntile + 1) / 2, kThreads, 0, st>>>((const float2*)O, d, w.winv, N, P, ntile,
                                                                       norm, w.K);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // z = K^-1 u (K overwritten by its Cholesky factor)
    e = launch_direct_solve(w.K, w.u, w.z, N, w.work, w.sync, res, st);
    if (e != cudaSuccess) return e;
    if (fp64)
        wb_cols<double2><<<gp, kThreads, 0, st>>>((const double2*)O, d, w.z, w.winv, w.y, N, P, x);
    else
        wb_cols<float2><<<gp, kThreads, 0, st>>>((const float2*)O, d, w.z, w.winv, w.y, N, P, x);
    return cudaGetLastError();
}

}  // namespace rbmnqs
