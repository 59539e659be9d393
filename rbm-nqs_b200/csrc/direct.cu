// direct.cu -- the direct SR solver (optimizer/direct_solver.cpp:31-59) on a
// formed S:
//
//   S_reg = S with its diagonal scaled by (1 + r1) ((1 + r1) + rd on the
//           non-neural parameters) + r2 max|diag| I,   S_reg x = F.
//
// The reference solves with Eigen's complete orthogonal decomposition.  S is
// a covariance matrix and the shift r2 max|diag| is positive, so S_reg is
// Hermitian positive definite and the solution is unique; it is computed
// here by a blocked Cholesky factorisation S_reg = L L^H and two triangular
// solves, FP64 throughout.
//
// One cooperative persistent kernel.  Per 32-column panel: block 0 factors
// the diagonal tile, every warp of the grid solves rows of the panel below
// it, and the blocks update the trailing lower triangle in 32 x 32 tiles.
// Grid barriers with bounded waits separate the phases (status
// RBMNQS_ERR_CUDA if one gives up).  A pivot that is not positive and
// finite marks the solve RBMNQS_ERR_NONFINITE; the factorisation continues
// with a unit pivot so that every block takes the same barriers.
#include <algorithm>

#include "coop.cuh"
#include "sr.cuh"

namespace rbmnqs {
namespace {

constexpr int kThreads = 256;
constexpr int kTile = 32;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 shfl2(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// A: P x P row-major, Hermitian (the lower triangle is read and overwritten
// by L).  y: P work entries.
__global__ void __launch_bounds__(kThreads) cholesky_solve_kernel(double2* A, int P, const double2* b, double2* x,
                                                                  double2* y, MfreeSync* sync, CgResultDev* res) {
    __shared__ double2 U[kTile][kTile + 1];
    __shared__ double2 V[kTile][kTile + 1];
    __shared__ int bad_pivot;
    const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
    const int nwb = kThreads / 32;
    const int gw = blockIdx.x * nwb + wib, nw = gridDim.x * nwb;
    const uint32_t G = gridDim.x;
    const int nb = (P + kTile - 1) / kTile;
    if (tid == 0) bad_pivot = 0;
    __syncthreads();
    bool ok = true;

    // ---- factorisation ----------------------------------------------------
    for (int K = 0; K < nb && ok; K++) {
        const int k0 = K * kTile, kw = min(kTile, P - k0);
        // (1) diagonal tile: unblocked right-looking Cholesky in shared memory
        if (blockIdx.x == 0) {
            for (int e = tid; e < kTile * kTile; e += kThreads) {
                const int i = e / kTile, j = e % kTile;
                U[i][j] = (i < kw && j <= i) ? __ldcg(A + (size_t)(k0 + i) * P + k0 + j) : make_double2(0, 0);
            }
            __syncthreads();
            for (int j = 0; j < kw; j++) {
                if (tid == 0) {
                    double dj = U[j][j].x;
                    if (!(dj > 0.0) || !isfinite(dj)) {
                        bad_pivot = 1;
                        dj = 1.0;
                    }
                    U[j][j] = make_double2(sqrt(dj), 0.0);
                }
                __syncthreads();
                const double ljj = U[j][j].x;
                for (int i = j + 1 + tid; i < kw; i += kThreads) U[i][j] = make_double2(U[i][j].x / ljj, U[i][j].y / ljj);
                __syncthreads();
                for (int e = tid; e < kTile * kTile; e += kThreads) {
                    const int i = e / kTile, l = e % kTile;
                    if (l > j && l <= i && i < kw) U[i][l] = csub(U[i][l], cmulc(U[i][j], U[l][j]));
                }
                __syncthreads();
            }
            for (int e = tid; e < kTile * kTile; e += kThreads) {
                const int i = e / kTile, j = e % kTile;
                if (i < kw && j <= i) A[(size_t)(k0 + i) * P + k0 + j] = U[i][j];
            }
        }
        if (!(ok = grid_barrier(sync, G))) break;
        // (2) the panel below: L21 L11^H = A21, one warp per row
        for (int e = tid; e < kTile * kTile; e += kThreads) {
            const int i = e / kTile, j = e % kTile;
            U[i][j] = (i < kw && j <= i) ? __ldcg(A + (size_t)(k0 + i) * P + k0 + j) : make_double2(0, 0);
        }
        __syncthreads();
        for (int i = k0 + kw + gw; i < P; i += nw) {
            double2 acc = lane < kw ? __ldcg(A + (size_t)i * P + k0 + lane) : make_double2(0, 0);
            for (int j = 0; j < kw; j++) {
                double2 xj = shfl2(acc, j);
                xj = make_double2(xj.x / U[j][j].x, xj.y / U[j][j].x);
                if (lane == j)
                    acc = xj;
                else if (lane > j)
                    acc = csub(acc, cmulc(xj, U[lane][j]));
            }
            if (lane < kw) A[(size_t)i * P + k0 + lane] = acc;
        }
        if (!(ok = grid_barrier(sync, G))) break;
        // (3) trailing update A22 -= L21 L21^H on the lower triangle, tile by tile
        const int m = nb - K - 1;
        const int ntiles = m * (m + 1) / 2;
        for (int t = blockIdx.x; t < ntiles; t += G) {
            int ip = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
            while ((ip + 1) * (ip + 2) / 2 <= t) ip++;
            while (ip * (ip + 1) / 2 > t) ip--;
            const int jp = t - ip * (ip + 1) / 2;
            const int I0 = (K + 1 + ip) * kTile, J0 = (K + 1 + jp) * kTile;
            const int ih = min(kTile, P - I0), jh = min(kTile, P - J0);
            __syncthreads();  // the previous tile's reads of U, V are done
            for (int e = tid; e < kTile * kTile; e += kThreads) {
                const int r = e / kTile, l = e % kTile;
                U[r][l] = (r < ih && l < kw) ? __ldcg(A + (size_t)(I0 + r) * P + k0 + l) : make_double2(0, 0);
                V[r][l] = (r < jh && l < kw) ? __ldcg(A + (size_t)(J0 + r) * P + k0 + l) : make_double2(0, 0);
            }
            __syncthreads();
            for (int e = tid; e < kTile * kTile; e += kThreads) {
                const int r = e / kTile, c = e % kTile;
                if (r < ih && c < jh && I0 + r >= J0 + c) {
                    double2 s = make_double2(0, 0);
                    for (int l = 0; l < kw; l++) {
                        const double2 p = cmulc(U[r][l], V[c][l]);
                        s.x += p.x;
                        s.y += p.y;
                    }
                    double2* a = A + (size_t)(I0 + r) * P + J0 + c;
                    *a = csub(__ldcg(a), s);
                }
            }
        }
        if (!(ok = grid_barrier(sync, G))) break;
    }

    // ---- L y = F --------------------------------------------------------------
    if (ok) {
        for (int i = blockIdx.x * kThreads + tid; i < P; i += G * kThreads) y[i] = b[i];
        ok = grid_barrier(sync, G);
    }
    for (int K = 0; K < nb && ok; K++) {
        const int k0 = K * kTile, kw = min(kTile, P - k0);
        if (blockIdx.x == 0 && wib == 0) {
            double2 acc = lane < kw ? __ldcg(y + k0 + lane) : make_double2(0, 0);
            for (int j = 0; j < kw; j++) {
                const double ljj = __ldcg(A + (size_t)(k0 + j) * P + k0 + j).x;
                double2 yj = shfl2(acc, j);
                yj = make_double2(yj.x / ljj, yj.y / ljj);
                if (lane == j)
                    acc = yj;
                else if (lane > j && lane < kw)
                    acc = csub(acc, cmul(__ldcg(A + (size_t)(k0 + lane) * P + k0 + j), yj));
            }
            if (lane < kw) y[k0 + lane] = acc;
        }
        if (!(ok = grid_barrier(sync, G))) break;
        for (int i = k0 + kw + gw; i < P; i += nw) {
            double2 s = make_double2(0, 0);
            if (lane < kw) s = cmul(__ldcg(A + (size_t)i * P + k0 + lane), __ldcg(y + k0 + lane));
            for (int o = 16; o; o >>= 1) {
                s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
                s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
            }
            if (lane == 0) y[i] = csub(__ldcg(y + i), s);
        }
        if (!(ok = grid_barrier(sync, G))) break;
    }

    // ---- L^H x = y ------------------------------------------------------------
    for (int K = nb - 1; K >= 0 && ok; K--) {
        const int k0 = K * kTile, kw = min(kTile, P - k0);
        if (blockIdx.x == 0 && wib == 0) {
            double2 acc = lane < kw ? __ldcg(y + k0 + lane) : make_double2(0, 0);
            for (int j = kw - 1; j >= 0; j--) {
                const double ljj = __ldcg(A + (size_t)(k0 + j) * P + k0 + j).x;
                double2 xj = shfl2(acc, j);
                xj = make_double2(xj.x / ljj, xj.y / ljj);
                if (lane == j)
                    acc = xj;
                else if (lane < j)
                    acc = csub(acc, cmulc(xj, __ldcg(A + (size_t)(k0 + j) * P + k0 + lane)));
            }
            if (lane < kw) x[k0 + lane] = acc;
        }
        if (!(ok = grid_barrier(sync, G))) break;
        if (k0 > 0) {
            if (tid < kTile) V[0][tid] = tid < kw ? __ldcg(x + k0 + tid) : make_double2(0, 0);
            __syncthreads();
            for (int i = blockIdx.x * kThreads + tid; i < k0; i += G * kThreads) {
                double2 s = make_double2(0, 0);
                for (int r = 0; r < kw; r++) {
                    const double2 p = cmulc(V[0][r], __ldcg(A + (size_t)(k0 + r) * P + i));
                    s.x += p.x;
                    s.y += p.y;
                }
                y[i] = csub(__ldcg(y + i), s);
            }
            __syncthreads();
        }
        if (!(ok = grid_barrier(sync, G))) break;
    }

    if (blockIdx.x == 0 && tid == 0) {
        res->iterations = 0;
        res->residual = 0;
        res->status = !ok ? -2 : (bad_pivot ? -5 : 0);
    }
}

}  // namespace

cudaError_t launch_direct_solve(double2* Sreg, const double2* F, double2* x, int P, double2* work, MfreeSync* sync,
                                CgResultDev* res, cudaStream_t st) {
    int dev = 0, per_sm = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cholesky_solve_kernel, kThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorLaunchOutOfResources;
    // enough blocks for the first trailing update, at most two per SM (the
    // barrier cost grows with the block count)
    const int nb = (P + kTile - 1) / kTile;
    const int tiles = (nb - 1) * nb / 2;
    const int blocks = std::max(1, std::min(tiles, std::min(per_sm, 2) * sms));
    e = launch_init_sync(sync, st);
    if (e != cudaSuccess) return e;
    void* args[] = {&Sreg, &P, (void*)&F, &x, &work, &sync, &res};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(cholesky_solve_kernel), dim3(blocks),
                                       dim3(kThreads), args, 0, st);
}

}  // namespace rbmnqs
