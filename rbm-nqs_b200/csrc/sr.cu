// sr.cu -- stochastic-reconfiguration kernels: sample moments, energy
// statistics, the Hermitian Gram S, regularisation, FP64 conjugate
// gradients and the weight update.
#include <cooperative_groups.h>

#include "common.cuh"
#include "sr.cuh"

namespace cgx = cooperative_groups;

namespace rbmnqs {

// ------------------------------------------------------- block reductions --
template <typename T> __device__ __forceinline__ T shfl_sum(T v);
template <> __device__ __forceinline__ double shfl_sum<double>(double v) { return warp_sum(v); }
template <> __device__ __forceinline__ double2 shfl_sum<double2>(double2 v) {
    v.x = warp_sum(v.x);
    v.y = warp_sum(v.y);
    return v;
}
__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// Deterministic block sum; every thread gets the result.  `red` must hold
// blockDim/32 entries.
template <typename T> __device__ T block_sum(T v, T* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = shfl_sum(v);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    T r = red[0];
    for (int i = 1; i < nw; i++) {
        if constexpr (sizeof(T) == 16) r = add2(r, red[i]);
        else r += red[i];
    }
    return r;
}

__device__ double block_max(double v, double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double r = red[0];
    for (int i = 1; i < nw; i++) r = fmax(r, red[i]);
    return r;
}

__device__ __forceinline__ double2 ld2(const float2* O, size_t i) {
    const float2 v = O[i];
    return make_double2(v.x, v.y);
}
__device__ __forceinline__ double2 ld2(const double2* O, size_t i) { return O[i]; }

// ------------------------------------------------------------- moments ---
// Per block over a slice of samples: sum_n O[n][p], sum_n E_n conj(O[n][p]),
// sum_n E_n (aggregators a_d_, a_dh_, a_h_: aggregator.cpp:190-231), each
// term weighted by w[n] when w is given (full enumeration, p = |psi|^2).
template <typename TO>
__global__ void moments_partial(const TO* O, const double2* E, int N, int P, double2* pd, double2* pf, double2* pe,
                                const double* w) {
    __shared__ double2 red[32];
    const int nb = gridDim.x;
    const int n0 = (int)((long)N * blockIdx.x / nb), n1 = (int)((long)N * (blockIdx.x + 1) / nb);
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        double sx = 0, sy = 0, fx = 0, fy = 0;
        auto add = [&](double2 o, int n) {
            if (w) {
                const double wn = w[n];
                o = make_double2(wn * o.x, wn * o.y);
            }
            const double2 e = E[n];
            sx += o.x;
            sy += o.y;
            fx += e.x * o.x + e.y * o.y;  // E * conj(O)
            fy += e.y * o.x - e.x * o.y;
        };
        // four rows' loads in flight before their (ordered) sums
        int n = n0;
        for (; n + 3 < n1; n += 4) {
            double2 o[4];
#pragma unroll
            for (int u = 0; u < 4; u++) o[u] = ld2(O, (size_t)(n + u) * P + p);
#pragma unroll
            for (int u = 0; u < 4; u++) add(o[u], n + u);
        }
        for (; n < n1; n++) add(ld2(O, (size_t)n * P + p), n);
        pd[(size_t)blockIdx.x * P + p] = make_double2(sx, sy);
        pf[(size_t)blockIdx.x * P + p] = make_double2(fx, fy);
    }
    double2 es = make_double2(0, 0);
    for (int n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
        const double2 e = E[n];
        es = add2(es, w ? make_double2(w[n] * e.x, w[n] * e.y) : e);
    }
    es = block_sum(es, red);
    if (threadIdx.x == 0) pe[blockIdx.x] = es;
}

// d = <O>, F = <E O*> - <E> conj(<O>) (stochastic_reconfiguration.cpp:102);
// the sums are divided by *wsum (the total weight) when given, else by N.
__global__ void moments_final(const double2* pd, const double2* pf, const double2* pe, int nb, int N_, int P,
                              double2* d, double2* F, double2* emean, const double* wsum) {
    // one warp per parameter, lanes over the partial blocks (fixed order)
    __shared__ double2 em;
    const double N = wsum ? *wsum : (double)N_;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    auto wsum2 = [&](double2 v) {
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_xor_sync(kFull, v.x, o);
            v.y += __shfl_xor_sync(kFull, v.y, o);
        }
        return v;
    };
    if (w == 0) {
        double2 s = make_double2(0, 0);
        for (int b = lane; b < nb; b += 32) s = add2(s, pe[b]);
        s = wsum2(s);
        if (lane == 0) {
            em = make_double2(s.x / N, s.y / N);
            if (blockIdx.x == 0) *emean = em;
        }
    }
    __syncthreads();
    for (int p = blockIdx.x * nw + w; p < P; p += gridDim.x * nw) {
        double2 sd = make_double2(0, 0), sf = make_double2(0, 0);
        for (int b = lane; b < nb; b += 32) {
            sd = add2(sd, pd[(size_t)b * P + p]);
            sf = add2(sf, pf[(size_t)b * P + p]);
        }
        sd = wsum2(sd);
        sf = wsum2(sf);
        if (lane == 0) {
            const double2 dd = make_double2(sd.x / N, sd.y / N);
            d[p] = dd;
            // F = dh - h * conj(d)
            F[p] = make_double2(sf.x / N - (em.x * dd.x + em.y * dd.y), sf.y / N - (em.y * dd.x - em.x * dd.y));
        }
    }
}

// ------------------------------------------------------ energy statistics --
// aggregator::finalize for a_h_ with n_bins bins (aggregator.cpp:84-164,
// 233-239): mean, M2, binned M2, tau, unbiased variances, binned stddev; and
// the mean acceptance over chains (metropolis_sampler.cpp:89-91).
// E_loc statistics of the epoch in one launch: block j of the n_bins blocks
// reads bin j (contiguous, coalesced) for its sum and its share of
// sum |e - mu|^2; the last block to finish adds the partials in bin order
// (deterministic) and writes the statistics.  part: 4 doubles per bin, then
// the ticket counter (zero between launches: the last block resets it).
__global__ void __launch_bounds__(256) energy_stats(const double2* E, int N, int n_bins, const double2* emean,
                                                    const uint32_t* nacc, const uint32_t* nprop, int n_chains,
                                                    double* part, EpochStatsDev* out) {
    __shared__ double red[32];
    __shared__ int last;
    unsigned int* ticket = reinterpret_cast<unsigned int*>(part + 4 * n_bins);
    const double2 mu = *emean;
    const int bs = N / n_bins;
    const double2* Eb = E + (size_t)blockIdx.x * bs;
    double m2 = 0, sx = 0, sy = 0;
    int finite = 1;
    for (int i = threadIdx.x; i < bs; i += blockDim.x) {
        const double2 e = Eb[i];
        if (!isfinite(e.x) || !isfinite(e.y)) finite = 0;
        const double dx = e.x - mu.x, dy = e.y - mu.y;
        m2 += dx * dx + dy * dy;
        sx += e.x;
        sy += e.y;
    }
    m2 = block_sum(m2, red);
    sx = block_sum(sx, red);
    sy = block_sum(sy, red);
    const double nf = block_sum((double)finite, red);
    if (threadIdx.x == 0) {
        double* pp = part + 4 * blockIdx.x;
        pp[0] = m2;
        pp[1] = sx;
        pp[2] = sy;
        pp[3] = nf == (double)blockDim.x ? 1.0 : 0.0;
        __threadfence();
        last = atomicAdd(ticket, 1u) == (unsigned int)(n_bins - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the partials into shared memory in parallel, then added in bin order
    __shared__ double sp[4 * kMaxBins];
    for (int i = threadIdx.x; i < 4 * n_bins; i += blockDim.x) sp[i] = reinterpret_cast<volatile double*>(part)[i];
    double acc = 0;
    for (int c = threadIdx.x; c < n_chains; c += blockDim.x) acc += nprop[c] ? (double)nacc[c] / nprop[c] : 0.0;
    acc = block_sum(acc, red);  // (its barriers also publish sp)
    if (threadIdx.x == 0) {
        double M2 = 0, M2b = 0;
        int fin = 1;
        for (int b = 0; b < n_bins; b++) {
            M2 += sp[4 * b];
            const double dx = sp[4 * b + 1] / bs - mu.x, dy = sp[4 * b + 2] / bs - mu.y;
            M2b += bs * (dx * dx + dy * dy);
            if (sp[4 * b + 3] == 0.0) fin = 0;
        }
        *ticket = 0u;
        double tau = 0;
        if (n_bins > 1 && !(M2 == 0 && M2b == 0)) {
            const double r = bs * M2b / M2;
            tau = 0.5 * ((r < 1 ? 1 : r) - 1);
        }
        const double den = (double)N - 1.0;
        double v = M2 / den, vb = M2b / den;
        v = v < 0 ? 0 : v;
        vb = vb < 0 ? 0 : vb;
        out->energy = mu;
        out->var = v;
        out->var_binned = vb;
        out->tau = tau;
        out->stddev = n_bins > 1 ? sqrt(vb / n_bins) : sqrt(v / N);
        out->acceptance = acc / n_chains;
        out->finite = fin;
    }
}

// ----------------------------------------------------------------- Gram ---
// S = (1/N) sum_n conj(X_n) X_n^T with X = O - <O> (centred, so no
// cancellation against conj(d) d^T).  FP64 accumulation of FP32/FP64 inputs
// on CUDA cores: 32x32 complex tiles of the upper triangle, split over
// sample ranges into partial buffers.
constexpr int GT = 32, GK = 16;

template <typename TO>
__global__ void __launch_bounds__(256) gram_fp64(const TO* O, const double2* d, int N, int P, int ntile,
                                                 double2* part) {
    __shared__ double2 A[GK][GT + 1];
    __shared__ double2 B[GK][GT + 1];
    // map blockIdx.x -> (tp <= tq)
    int t = blockIdx.x, tp = 0;
    while (t >= ntile - tp) {
        t -= ntile - tp;
        tp++;
    }
    const int tq = tp + t;
    const int p0 = tp * GT, q0 = tq * GT;
    const int ks = blockIdx.y, nks = gridDim.y;
    const int n0 = (int)((long)N * ks / nks), n1 = (int)((long)N * (ks + 1) / nks);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double2 acc[2][2];
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) acc[i][j] = make_double2(0, 0);
    for (int nb = n0; nb < n1; nb += GK) {
        for (int i = threadIdx.x; i < GK * GT; i += blockDim.x) {
            const int kk = i / GT, c = i % GT;
            const int n = nb + kk;
            double2 a = make_double2(0, 0), b = make_double2(0, 0);
            if (n < n1) {
                if (p0 + c < P) {
                    a = ld2(O, (size_t)n * P + p0 + c);
                    if (d) {
                        a.x -= d[p0 + c].x;
                        a.y -= d[p0 + c].y;
                    }
                }
                if (q0 + c < P) {
                    b = ld2(O, (size_t)n * P + q0 + c);
                    if (d) {
                        b.x -= d[q0 + c].x;
                        b.y -= d[q0 + c].y;
                    }
                }
            }
            A[kk][c] = a;
            B[kk][c] = b;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk++) {
            const double2 a0 = A[kk][ty], a1 = A[kk][ty + 16];
            const double2 b0 = B[kk][tx], b1 = B[kk][tx + 16];
            const double2 av[2] = {a0, a1}, bv[2] = {b0, b1};
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    // conj(a) * b
                    acc[i][j].x = fma(av[i].x, bv[j].x, fma(av[i].y, bv[j].y, acc[i][j].x));
                    acc[i][j].y = fma(av[i].x, bv[j].y, fma(-av[i].y, bv[j].x, acc[i][j].y));
                }
        }
        __syncthreads();
    }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            const int p = p0 + ty + 16 * i, q = q0 + tx + 16 * j;
            if (p < P && q < P) part[(size_t)ks * P * P + (size_t)p * P + q] = acc[i][j];
        }
}

// Sum the split partials, scale by 1/N, mirror the lower triangle.
__global__ void gram_finalize(const double2* part, int nks, int N, int P, double2* S) {
    const size_t total = (size_t)P * P;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int p = (int)(i / P), q = (int)(i % P);
        if (q < p) continue;
        double2 s = make_double2(0, 0);
        for (int k = 0; k < nks; k++) s = add2(s, part[(size_t)k * total + i]);
        s.x /= N;
        s.y /= N;
        if (p == q) s.y = 0;
        S[i] = s;
        S[(size_t)q * P + p] = make_double2(s.x, -s.y);
    }
}

// ------------------------------------------------------ schedule / reg ---
// decay_t::get for the four schedules (abstract_optimizer.cpp:27-54).
__global__ void schedule_step(ScheduleDev* s, int first) {
    if (threadIdx.x >= first && threadIdx.x < 4) {
        const int i = threadIdx.x;
        if (!s->min_reached[i]) {
            s->value[i] *= s->decay[i];
            if (s->value[i] < s->min[i]) {
                s->min_reached[i] = 1;
                s->value[i] = s->min[i];
            }
        }
    }
}

// diag = var(O) = N/(N-1) S_pp; S_reg = S + r1 diag (+ rd on non-neural
// parameters) + r2 max(diag) (cg_solver.cpp:301-318).  direct: S_pp (1 + r1)
// ((1 + r1) + rd on non-neural parameters) + r2 max|diag|
// (direct_solver.cpp:42-49).
__global__ void regularize(const double2* S, int P, int n_neural, int N, const ScheduleDev* sch, double* diag,
                           double2* Sreg, double* max_diag_out, int direct, const double* vfac) {
    __shared__ double red[32];
    const double r1 = sch->value[1], r2 = sch->value[2], rd = sch->value[3];
    // unbiased variance factor: N / (N - 1), or W / (W - W2 / W) for weights
    const double vf = vfac ? *vfac : (double)N / ((double)N - 1.0);
    // every block forms max(diag) itself (order-free); block 0 stores diag
    double mx = 0;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const double v = S[(size_t)p * P + p].x * vf;
        if (blockIdx.x == 0) diag[p] = v;
        mx = fmax(mx, v);
    }
    mx = block_max(mx, red);
    if (blockIdx.x == 0 && threadIdx.x == 0) *max_diag_out = mx;
    // the copy over all blocks, the shift applied to the diagonal entries
    // (index p (P + 1)) on the way
    const size_t total = (size_t)P * P;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        double2 s = S[i];
        if (i % (size_t)(P + 1) == 0) {
            const int p = (int)(i / (size_t)(P + 1));
            if (direct) {
                const double g = p < n_neural ? 1.0 + r1 : (1.0 + r1) + rd;
                s = make_double2(s.x * g + r2 * mx, s.y * g);
            } else {
                s.x += s.x * vf * (p < n_neural ? r1 : r1 + rd) + mx * r2;
            }
        }
        Sreg[i] = s;
    }
}

// abstract_solver::solve inputs (drop-in entry point): S_reg = G/norm -
// conj(d) d^T + diag(r1 diag (+rd) + r2 max(diag)), where G = sum conj(O) O^T
// was accumulated with weights already folded into O (cg_solver.cpp:301-318).
__global__ void solve_prep(const double2* G, int N, double norm, const double2* d, const double* diag, int P,
                           int n_neural, double r1, double r2, double rd, double2* Sreg, int direct) {
    __shared__ double red[32];
    double mx = -1e300;
    for (int p = threadIdx.x; p < P; p += blockDim.x) mx = fmax(mx, diag[p]);
    mx = block_max(mx, red);
    const double scale = (double)N / norm;  // G holds sums divided by N
    const size_t total = (size_t)P * P;
    for (size_t i = threadIdx.x; i < total; i += blockDim.x) {
        const int k = (int)(i / P), l = (int)(i % P);
        const double2 g = G[i], dk = d[k], dl = d[l];
        // conj(d_k) d_l
        const double cx = dk.x * dl.x + dk.y * dl.y, cy = dk.x * dl.y - dk.y * dl.x;
        double2 v = make_double2(g.x * scale - cx, g.y * scale - cy);
        if (k == l) {
            if (direct) {
                const double gk = k < n_neural ? 1.0 + r1 : (1.0 + r1) + rd;
                v = make_double2(v.x * gk + r2 * mx, v.y * gk);
            } else {
                v.x += diag[k] * (k < n_neural ? r1 : r1 + rd) + mx * r2;
            }
        }
        Sreg[i] = v;
    }
}

cudaError_t launch_solve_prep(const double2* G, int N, double norm, const double2* d, const double* diag, int P,
                              int n_neural, double r1, double r2, double rd, double2* Sreg, cudaStream_t st,
                              int direct) {
    solve_prep<<<1, 1024, 0, st>>>(G, N, norm, d, diag, P, n_neural, r1, r2, rd, Sreg, direct);
    return cudaGetLastError();
}

// -------------------------------------------------------------------- CG --
// cg_solver::cg1 (cg_solver.cpp:119-193) on the dense regularised S, one
// block; vectors in shared memory.  Stops when ||r||^2 < rtol or after
// max_it iterations.
__global__ void __launch_bounds__(1024) cg_dense(const double2* A, const double2* b, double2* x, int P, int max_it,
                                                 double rtol, CgResultDev* res) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2* r = reinterpret_cast<double2*>(sm);
    double2* p = r + P;
    double2* Ap = p + P;
    __shared__ double red[32];
    __shared__ double2 red2[32];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
    auto matvec = [&](const double2* v) {
        for (int row = w; row < P; row += nw) {
            double sx = 0, sy = 0;
            const double2* Ar = A + (size_t)row * P;
            for (int j = lane; j < P; j += 32) {
                const double2 a = Ar[j], vv = v[j];
                sx = fma(a.x, vv.x, fma(-a.y, vv.y, sx));
                sy = fma(a.x, vv.y, fma(a.y, vv.x, sy));
            }
            sx = warp_sum(sx);
            sy = warp_sum(sy);
            if (lane == 0) Ap[row] = make_double2(sx, sy);
        }
        __syncthreads();
    };
    for (int i = tid; i < P; i += nt) p[i] = x[i];
    __syncthreads();
    matvec(p);
    double rs0 = 0;
    for (int i = tid; i < P; i += nt) {
        const double2 ri = make_double2(b[i].x - Ap[i].x, b[i].y - Ap[i].y);
        r[i] = ri;
        p[i] = ri;
        rs0 += ri.x * ri.x + ri.y * ri.y;
    }
    double rsold = block_sum(rs0, red);
    double rs = rsold;
    int itn = 0;
    for (itn = 0; itn < max_it; itn++) {
        matvec(p);
        double2 pap = make_double2(0, 0);
        for (int i = tid; i < P; i += nt) {  // p^H Ap
            pap.x += p[i].x * Ap[i].x + p[i].y * Ap[i].y;
            pap.y += p[i].x * Ap[i].y - p[i].y * Ap[i].x;
        }
        pap = block_sum(pap, red2);
        // alpha = rsold / pap
        const double den = pap.x * pap.x + pap.y * pap.y;
        const double ax = rsold * pap.x / den, ay = -rsold * pap.y / den;
        double rl = 0;
        for (int i = tid; i < P; i += nt) {
            const double2 pi = p[i], api = Ap[i];
            double2 xi = x[i];
            xi.x += ax * pi.x - ay * pi.y;
            xi.y += ax * pi.y + ay * pi.x;
            x[i] = xi;
            double2 ri = r[i];
            ri.x -= ax * api.x - ay * api.y;
            ri.y -= ax * api.y + ay * api.x;
            r[i] = ri;
            rl += ri.x * ri.x + ri.y * ri.y;
        }
        rs = block_sum(rl, red);
        if (rs < rtol) break;
        const double beta = rs / rsold;
        for (int i = tid; i < P; i += nt) {
            const double2 ri = r[i], pi = p[i];
            p[i] = make_double2(ri.x + beta * pi.x, ri.y + beta * pi.y);
        }
        rsold = rs;
        __syncthreads();
    }
    if (tid == 0) {
        res->iterations = itn;
        res->residual = rs;
    }
}

// Same iteration with S_reg resident in shared memory as its packed upper
// triangle (row i holds S_ij, j >= i, at off(i) + j - i with
// off(i) = i P - i(i-1)/2; S_ji = conj(S_ij)).  Fits for P <= 157.
// Work split: 8 lanes per matrix row (each lane ~P/8 complex MACs, a 3-level
// shuffle finishes the row); p^H Ap is accumulated in the matvec epilogue;
// block sums go through one partial per warp reduced with shuffles, so one
// iteration costs three barriers.
__host__ __device__ inline size_t packed_size(int P) { return (size_t)P * (P + 1) / 2; }

__device__ __forceinline__ double2 shfl_xor2(double2 v, int o) {
    return make_double2(__shfl_xor_sync(kFull, v.x, o), __shfl_xor_sync(kFull, v.y, o));
}

// Sum of the per-warp partials part[0..nw) seen by every thread.
__device__ __forceinline__ double2 sum_partials2(const double2* part, int nw) {
    const int lane = threadIdx.x & 31;
    double2 v = lane < nw ? part[lane] : make_double2(0, 0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double2 w = shfl_xor2(v, o);
        v.x += w.x;
        v.y += w.y;
    }
    return v;
}

__global__ void __launch_bounds__(1024) cg_packed(const double2* A, const double2* b, double2* xg, int P, int max_it,
                                                  double rtol, CgResultDev* res) {
    extern __shared__ __align__(16) unsigned char sm[];
    double2* U = reinterpret_cast<double2*>(sm);
    double2* r = U + packed_size(P);
    double2* p = r + P;
    double2* Ap = p + P;
    double2* x = Ap + P;
    __shared__ double2 partA[32], partB[32];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
    const int sub = lane & 7;  // lane within the 8-lane row group
    for (int i = w; i < P; i += nw) {
        const size_t o = (size_t)i * P - (size_t)i * (i - 1) / 2;
        for (int j = i + lane; j < P; j += 32) U[o + j - i] = A[(size_t)i * P + j];
    }
    for (int i = tid; i < P; i += nt) {
        x[i] = xg[i];
        p[i] = xg[i];
    }
    __syncthreads();
    // Ap = A p; returns this thread's share of p^H Ap (summed over rows it
    // finished), caller reduces
    auto matvec = [&]() -> double2 {
        double2 pap = make_double2(0, 0);
        // warp-uniform trip count: warp w covers rows r0 .. r0+3 of each
        // block of 4 * nw rows; lanes of rows >= P compute nothing but still
        // join every shuffle
        for (int r0 = 4 * w; r0 < P; r0 += 4 * nw) {
            const int row = r0 + (lane >> 3);
            const bool ok = row < P;
            double sx = 0, sy = 0;
            if (ok) {
                const size_t orow = (size_t)row * P - (size_t)row * (row - 1) / 2;
                for (int j = sub; j < P; j += 8) {
                    double2 a;
                    if (j >= row) {
                        a = U[orow + j - row];
                    } else {
                        const double2 t = U[(size_t)j * P - (size_t)j * (j - 1) / 2 + row - j];
                        a = make_double2(t.x, -t.y);
                    }
                    const double2 vv = p[j];
                    sx = fma(a.x, vv.x, fma(-a.y, vv.y, sx));
                    sy = fma(a.x, vv.y, fma(a.y, vv.x, sy));
                }
            }
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) {
                sx += __shfl_xor_sync(kFull, sx, o);
                sy += __shfl_xor_sync(kFull, sy, o);
            }
            if (ok && sub == 0) {
                Ap[row] = make_double2(sx, sy);
                const double2 pr = p[row];
                pap.x += pr.x * sx + pr.y * sy;  // conj(p) * Ap
                pap.y += pr.x * sy - pr.y * sx;
            }
        }
        return pap;
    };
    auto warp_total2 = [&](double2 v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double2 t = shfl_xor2(v, o);
            v.x += t.x;
            v.y += t.y;
        }
        return v;
    };
    (void)matvec();
    __syncthreads();
    double rs0 = 0;
    for (int i = tid; i < P; i += nt) {
        const double2 ri = make_double2(b[i].x - Ap[i].x, b[i].y - Ap[i].y);
        r[i] = ri;
        p[i] = ri;
        rs0 += ri.x * ri.x + ri.y * ri.y;
    }
    {
        const double2 t = warp_total2(make_double2(rs0, 0));
        if (lane == 0) partB[w] = t;
    }
    __syncthreads();
    double rsold = sum_partials2(partB, nw).x;
    double rs = rsold;
    int itn = 0;
    for (itn = 0; itn < max_it; itn++) {
        // (1) Ap = A p and p^H Ap
        {
            const double2 t = warp_total2(matvec());
            if (lane == 0) partA[w] = t;
        }
        __syncthreads();
        // (2) alpha, x += alpha p, r -= alpha Ap, ||r||^2
        const double2 pap = sum_partials2(partA, nw);
        const double den = pap.x * pap.x + pap.y * pap.y;
        const double ax = rsold * pap.x / den, ay = -rsold * pap.y / den;
        double rl = 0;
        for (int i = tid; i < P; i += nt) {
            const double2 pi = p[i], api = Ap[i];
            double2 xi = x[i];
            xi.x += ax * pi.x - ay * pi.y;
            xi.y += ax * pi.y + ay * pi.x;
            x[i] = xi;
            double2 ri = r[i];
            ri.x -= ax * api.x - ay * api.y;
            ri.y -= ax * api.y + ay * api.x;
            r[i] = ri;
            rl += ri.x * ri.x + ri.y * ri.y;
        }
        {
            const double2 t = warp_total2(make_double2(rl, 0));
            if (lane == 0) partB[w] = t;
        }
        __syncthreads();
        // (3) convergence test and p = r + beta p
        rs = sum_partials2(partB, nw).x;
        if (rs < rtol) break;
        const double beta = rs / rsold;
        for (int i = tid; i < P; i += nt) {
            const double2 ri = r[i], pi = p[i];
            p[i] = make_double2(ri.x + beta * pi.x, ri.y + beta * pi.y);
        }
        rsold = rs;
        __syncthreads();
    }
    for (int i = tid; i < P; i += nt) xg[i] = x[i];
    if (tid == 0) {
        res->iterations = itn;
        res->residual = rs;
    }
}

// The same iteration spread over one thread-block cluster of kClusterCta
// CTAs on as many SMs.  CTA c owns rows [c*rp, (c+1)*rp) of S_reg (full rows
// in its shared memory) and the matching slices of x, Ap; every CTA keeps
// full copies of p and r.  Per iteration: local mat-vec and p^H Ap partial,
// partial pushed into every CTA's shared memory (DSMEM store), cluster
// barrier; alpha, x/r update of the own rows, the new r rows and the
// ||r||^2 partial pushed to every CTA, barrier; beta and the whole new p
// computed by every CTA from its full r and p (the same arithmetic on the
// same data in every CTA, so the copies agree).  Two cluster barriers per
// iteration.  The operator, the arithmetic order within a row and the
// stopping rule are those of cg_packed.
constexpr int kClusterCta = 8;

__global__ void __cluster_dims__(kClusterCta, 1, 1) __launch_bounds__(256)
    cg_cluster(const double2* A, const double2* b, double2* xg, int P, int max_it, double rtol, CgResultDev* res) {
    extern __shared__ __align__(16) unsigned char sm[];
    cgx::cluster_group cl = cgx::this_cluster();
    const int rank = (int)cl.block_rank();
    const int rp = (P + kClusterCta - 1) / kClusterCta;
    const int r0 = rank * rp, r1 = min(P, r0 + rp), nr = max(0, r1 - r0);
    double2* Srow = reinterpret_cast<double2*>(sm);  // [rp][P]
    double2* p = Srow + (size_t)rp * P;              // [P] full copy
    double2* x = p + P;                              // [rp]
    double2* rf = x + rp;                            // [P] full copy of r
    double2* Ap = rf + P;                            // [rp]
    __shared__ double2 partA[kClusterCta], partB[kClusterCta];
    __shared__ double2 wred[8];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
    const int sub = lane & 7;
    for (int i = tid; i < nr * P; i += nt) Srow[i] = A[(size_t)r0 * P + i];
    for (int i = tid; i < P; i += nt) p[i] = xg[i];
    for (int i = tid; i < nr; i += nt) x[i] = xg[r0 + i];
    __syncthreads();

    auto cta_sum = [&](double2 v) -> double2 {  // every thread gets the CTA total
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_xor_sync(kFull, v.x, o);
            v.y += __shfl_xor_sync(kFull, v.y, o);
        }
        __syncthreads();
        if (lane == 0) wred[w] = v;
        __syncthreads();
        double2 t = make_double2(0, 0);
        for (int i = 0; i < nw; i++) {
            t.x += wred[i].x;
            t.y += wred[i].y;
        }
        return t;
    };
    // push this CTA's partial into slot `rank` of every CTA's array
    auto push = [&](double2* arr, double2 v) {
        if (tid < kClusterCta) {
            double2* dst = cl.map_shared_rank(arr, tid);
            dst[rank] = v;
        }
    };
    auto total = [&](const double2* arr) {
        double2 t = make_double2(0, 0);
        for (int i = 0; i < kClusterCta; i++) {
            t.x += arr[i].x;
            t.y += arr[i].y;
        }
        return t;
    };
    // local rows of A p; returns this thread's share of p^H Ap
    auto matvec = [&]() -> double2 {
        double2 pap = make_double2(0, 0);
        for (int q0 = 4 * w; q0 < nr; q0 += 4 * nw) {
            const int q = q0 + (lane >> 3);
            const bool ok = q < nr;
            double sx = 0, sy = 0;
            if (ok) {
                const double2* Ar = Srow + (size_t)q * P;
                for (int j = sub; j < P; j += 8) {
                    const double2 a = Ar[j], vv = p[j];
                    sx = fma(a.x, vv.x, fma(-a.y, vv.y, sx));
                    sy = fma(a.x, vv.y, fma(a.y, vv.x, sy));
                }
            }
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) {
                sx += __shfl_xor_sync(kFull, sx, o);
                sy += __shfl_xor_sync(kFull, sy, o);
            }
            if (ok && sub == 0) {
                Ap[q] = make_double2(sx, sy);
                const double2 pr = p[r0 + q];
                pap.x += pr.x * sx + pr.y * sy;
                pap.y += pr.x * sy - pr.y * sx;
            }
        }
        return pap;
    };

    (void)matvec();
    __syncthreads();
    double rl0 = 0;
    for (int i = tid; i < nr; i += nt) {
        const double2 ri = make_double2(b[r0 + i].x - Ap[i].x, b[r0 + i].y - Ap[i].y);
        for (int c = 0; c < kClusterCta; c++) cl.map_shared_rank(rf, c)[r0 + i] = ri;
        rl0 += ri.x * ri.x + ri.y * ri.y;
    }
    push(partB, cta_sum(make_double2(rl0, 0)));
    cl.sync();  // all of r is in every CTA; every CTA has finished reading p = x0
    for (int i = tid; i < P; i += nt) p[i] = rf[i];  // p = r
    __syncthreads();
    double rsold = total(partB).x;
    double rs = rsold;
    int itn = 0;
    for (itn = 0; itn < max_it; itn++) {
        push(partA, cta_sum(matvec()));
        cl.sync();
        const double2 pap = total(partA);
        const double den = pap.x * pap.x + pap.y * pap.y;
        const double ax = rsold * pap.x / den, ay = -rsold * pap.y / den;
        double rl = 0;
        for (int i = tid; i < nr; i += nt) {
            const double2 pi = p[r0 + i], api = Ap[i];
            double2 xi = x[i];
            xi.x += ax * pi.x - ay * pi.y;
            xi.y += ax * pi.y + ay * pi.x;
            x[i] = xi;
            double2 ri = rf[r0 + i];
            ri.x -= ax * api.x - ay * api.y;
            ri.y -= ax * api.y + ay * api.x;
            for (int c = 0; c < kClusterCta; c++) cl.map_shared_rank(rf, c)[r0 + i] = ri;
            rl += ri.x * ri.x + ri.y * ri.y;
        }
        push(partB, cta_sum(make_double2(rl, 0)));
        cl.sync();  // the new r is complete in every CTA
        rs = total(partB).x;
        if (rs < rtol) break;
        const double beta = rs / rsold;
        for (int i = tid; i < P; i += nt) {
            const double2 ri = rf[i], pi = p[i];
            p[i] = make_double2(ri.x + beta * pi.x, ri.y + beta * pi.y);
        }
        rsold = rs;
        __syncthreads();
    }
    for (int i = tid; i < nr; i += nt) xg[r0 + i] = x[i];
    if (rank == 0 && tid == 0) {
        res->iterations = itn;
        res->residual = rs;
    }
    cl.sync();  // no CTA leaves while others may still write its memory
}

// ---------------------------------------------------------------- update --
// abstract_optimizer::optimize tail (abstract_optimizer.cpp:150-177): the
// max|dw| > 30 guard, then the plugin (plugin.cpp:43-85) or dw *= lr, then
// w -= dw (rbm_base.cpp:117-131).  x keeps dw as the next warm start.
__global__ void sr_update(double2* params, double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                          PluginDev* plug) {
    __shared__ double red[32];
    if (res->status == -2) return;  // the solve itself failed (matrix-free CG barrier timeout)
    double mx = 0;
    int bad = 0;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const double2 v = x[i];
        if (!isfinite(v.x) || !isfinite(v.y)) bad = 1;
        mx = fmax(mx, sqrt(v.x * v.x + v.y * v.y));
    }
    mx = block_max(mx, red);
    const double nbad = block_sum((double)bad, red);
    const int status = nbad > 0 ? -5 : (mx > 30.0 ? -4 : 0);
    if (threadIdx.x == 0) {
        res->max_dw = mx;
        res->status = status;
    }
    // a non-finite direction is no warm start for the next solve (the
    // reference stops the run here, main.cpp:610-615)
    if (status == -5)
        for (int i = threadIdx.x; i < P; i += blockDim.x) x[i] = make_double2(0.0, 0.0);
    if (status != 0) return;
    const double lr = sch->value[0];
    const int type = plug ? plug->type : 0;
    if (type == 1) {
        // adam_plugin::apply: second moment split into real and imaginary parts
        const int t = plug->t;
        const double b1 = plug->beta1, b2 = plug->beta2, eps = plug->eps;
        const double c1 = 1.0 - pow(b1, (double)t), c2 = 1.0 - pow(b2, (double)t);
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
            const double2 g = x[i];
            double2 m = plug->m[i];
            m = make_double2(b1 * m.x + (1 - b1) * g.x, b1 * m.y + (1 - b1) * g.y);
            const double wr = b2 * plug->wr[i] + (1 - b2) * g.x * g.x;
            const double wi = b2 * plug->wi[i] + (1 - b2) * g.y * g.y;
            plug->m[i] = m;
            plug->wr[i] = wr;
            plug->wi[i] = wi;
            x[i] = make_double2((m.x / c1) / (sqrt(wr / c2) + eps) * lr, (m.y / c1) / (sqrt(wi / c2) + eps) * lr);
        }
        __syncthreads();
        if (threadIdx.x == 0) plug->t = t + 1;
    } else if (type == 2) {
        // momentum_plugin::apply: a momentum that is zero (every |m_i| <=
        // 1e-12, Eigen's isZero) starts at dw
        double nz = 0;
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
            const double2 m = plug->m[i];
            if (m.x * m.x + m.y * m.y > 1e-24) nz = 1;
        }
        nz = block_max(nz, red);
        double ax = plug->alpha;
        const double dup = plug->dup;
        double dnew = dup;
        if (dup < 1.0) {
            dnew = dup * plug->dialup;
            ax *= dnew;
        }
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
            const double2 g = x[i];
            const double2 m0 = nz > 0 ? plug->m[i] : g;
            const double2 m = make_double2(ax * m0.x + (1 - ax) * g.x, ax * m0.y + (1 - ax) * g.y);
            plug->m[i] = m;
            x[i] = make_double2(lr * m.x, lr * m.y);
        }
        __syncthreads();
        if (threadIdx.x == 0) plug->dup = dnew;
    } else {
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
            double2 v = x[i];
            v.x *= lr;
            v.y *= lr;
            x[i] = v;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const double2 v = x[i];
        params[i].x -= v.x;
        params[i].y -= v.y;
    }
}

// ------------------------------------------------------------------ heun --
// heun_plugin::apply (plugin.cpp:87-115).  The first step guards x1 like
// abstract_optimizer::optimize (abstract_optimizer.cpp:157), then moves the
// weights by delta = (lr/2) x1 without counting an update (update_weights_nc).
__global__ void heun_begin(double2* params, const double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                           PluginDev* plug) {
    __shared__ double red[32];
    if (res->status == -2) {
        if (threadIdx.x == 0) plug->gstat = -2;
        return;
    }
    double mx = 0;
    int bad = 0;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const double2 v = x[i];
        if (!isfinite(v.x) || !isfinite(v.y)) bad = 1;
        mx = fmax(mx, sqrt(v.x * v.x + v.y * v.y));
    }
    mx = block_max(mx, red);
    const double nbad = block_sum((double)bad, red);
    const int status = nbad > 0 ? -5 : (mx > 30.0 ? -4 : 0);
    if (threadIdx.x == 0) {
        res->max_dw = mx;
        res->status = status;
        plug->gstat = status;
        plug->gmax = mx;
    }
    if (status != 0) return;
    const double hl = 0.5 * sch->value[0];
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const double2 v = x[i];
        const double2 dl = make_double2(hl * v.x, hl * v.y);
        plug->m[i] = dl;
        params[i].x -= dl.x;
        params[i].y -= dl.y;
    }
}

// delta = (delta - (lr/2) x2) / 6; dd = d^T delta (no conjugate); |delta|^2.
__global__ void heun_delta(const double2* x, int P, const ScheduleDev* sch, const double2* d, PluginDev* plug) {
    __shared__ double red[32];
    if (plug->gstat != 0) return;
    const double hl = 0.5 * sch->value[0];
    double ddr = 0, ddi = 0, n2 = 0;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const double2 v = x[i];
        const double2 m = plug->m[i];
        const double2 dl = make_double2((m.x - hl * v.x) / 6.0, (m.y - hl * v.y) / 6.0);
        plug->m[i] = dl;
        if (d) {
            const double2 a = d[i];
            ddr += a.x * dl.x - a.y * dl.y;
            ddi += a.x * dl.y + a.y * dl.x;
        }
        n2 += dl.x * dl.x + dl.y * dl.y;
    }
    ddr = block_sum(ddr, red);
    ddi = block_sum(ddi, red);
    n2 = block_sum(n2, red);
    if (threadIdx.x == 0) {
        plug->dd = make_double2(ddr, ddi);
        plug->nrm2 = n2;
    }
}

// Per block: sum over its samples s of |sum_k delta_k O_sk - dd|^2 (the
// metric of the SR plugin hook, stochastic_reconfiguration.cpp:111-113).
// One warp per sample; sample-major O [N][P].
template <typename TO>
__global__ void heun_metric(const TO* O, int N, int P, PluginDev* plug) {
    __shared__ double red[32];
    if (plug->gstat != 0) return;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double2* dl = plug->m;
    const double2 dd = plug->dd;
    double acc = 0;
    for (int sIdx = blockIdx.x * nw + wib; sIdx < N; sIdx += gridDim.x * nw) {
        const TO* row = O + (size_t)sIdx * P;
        double er = 0, ei = 0;
        for (int k = lane; k < P; k += 32) {
            const TO o = row[k];
            const double2 a = dl[k];
            er += a.x * (double)o.x - a.y * (double)o.y;
            ei += a.x * (double)o.y + a.y * (double)o.x;
        }
        for (int off = 16; off; off >>= 1) {
            er += __shfl_xor_sync(0xffffffffu, er, off);
            ei += __shfl_xor_sync(0xffffffffu, ei, off);
        }
        er -= dd.x;
        ei -= dd.y;
        acc += er * er + ei * ei;  // identical in every lane
    }
    if (lane != 0) acc = 0;
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) plug->part[blockIdx.x] = acc;
}

// err = sqrt(sum)/P (SR metric) or |delta| (SGD); dw = x2 (cbrt-like factor)
__global__ void heun_end(double2* params, double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                         PluginDev* plug, int metric) {
    if (plug->gstat != 0) {
        if (threadIdx.x == 0) {
            res->status = plug->gstat;
            res->max_dw = plug->gmax;
        }
        return;
    }
    if (res->status == -2) return;  // the second solve failed
    double err;
    if (metric) {
        double sm = 0;
        for (int b = 0; b < kHeunBlocks; b++) sm += plug->part[b];  // fixed order
        err = sqrt(sm) / (double)P;
    } else {
        err = sqrt(plug->nrm2);
    }
    const double xx = pow(plug->heps / err, 1.0 / 3.0);
    const double f = (xx - 0.5) * sch->value[0];
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        double2 v = x[i];
        v.x *= f;
        v.y *= f;
        x[i] = v;
        params[i].x -= v.x;
        params[i].y -= v.y;
    }
    if (threadIdx.x == 0) {
        res->status = 0;
        res->max_dw = plug->gmax;
    }
}

cudaError_t launch_heun_begin(double2* params, const double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                              PluginDev* plug, cudaStream_t st) {
    heun_begin<<<1, 1024, 0, st>>>(params, x, P, sch, res, plug);
    return cudaGetLastError();
}

cudaError_t launch_heun_finish(double2* params, double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                               PluginDev* plug, const void* O, int fp64, const double2* d, int N, int metric,
                               cudaStream_t st) {
    heun_delta<<<1, 1024, 0, st>>>(x, P, sch, metric ? d : nullptr, plug);
    if (metric) {
        if (fp64)
            heun_metric<double2><<<kHeunBlocks, 256, 0, st>>>(static_cast<const double2*>(O), N, P, plug);
        else
            heun_metric<float2><<<kHeunBlocks, 256, 0, st>>>(static_cast<const float2*>(O), N, P, plug);
    }
    heun_end<<<1, 1024, 0, st>>>(params, x, P, sch, res, plug, metric);
    return cudaGetLastError();
}

// Parameter vector -> kernel layouts (site-major W in FP64 and FP32).
__global__ void unpack_weights(const double2* params, int n, int n_vb, int nh, double2* vb, double2* hb, double2* W64,
                               float2* W32) {
    const int tot = n * nh;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < tot + nh + n_vb; i += gridDim.x * blockDim.x) {
        if (i < n_vb) {
            vb[i] = params[i];
        } else if (i < n_vb + nh) {
            hb[i - n_vb] = params[i];
        } else {
            const int r = i - n_vb - nh;  // reference index j + n*k
            const int j = r % n, k = r / n;
            const double2 w = params[i];
            W64[j * nh + k] = w;
            W32[j * nh + k] = make_float2((float)w.x, (float)w.y);
        }
    }
}

// ---------------------------------------------------------------- launch --
cudaError_t launch_moments(const void* O, int fp64, const double2* E, int N, int P, int nblk, double2* pd,
                           double2* pf, double2* pe, double2* d, double2* F, double2* emean, cudaStream_t st,
                           const double* w, const double* wsum) {
    // one column per thread (a single pass over the block's rows) up to 1024
    // parameters
    const int thr = std::min(1024, std::max(32, (P + 31) / 32 * 32));
    if (fp64)
        moments_partial<double2><<<nblk, thr, 0, st>>>((const double2*)O, E, N, P, pd, pf, pe, w);
    else
        moments_partial<float2><<<nblk, thr, 0, st>>>((const float2*)O, E, N, P, pd, pf, pe, w);
    moments_final<<<(P + 7) / 8, 256, 0, st>>>(pd, pf, pe, nblk, N, P, d, F, emean, wsum);
    return cudaGetLastError();
}

// mean of E[N] (complex) into *mu, one block
__global__ void cmean_kernel(const double2* E, int N, double2* mu) {
    __shared__ double2 red[32];
    double2 s = make_double2(0, 0);
    for (int i = threadIdx.x; i < N; i += blockDim.x) s = add2(s, E[i]);
    s = block_sum(s, red);
    if (threadIdx.x == 0) *mu = make_double2(s.x / N, s.y / N);
}

cudaError_t launch_mean(const double2* E, int N, double2* mu, cudaStream_t st) {
    cmean_kernel<<<1, 1024, 0, st>>>(E, N, mu);
    return cudaGetLastError();
}

cudaError_t launch_energy_stats(const double2* E, int N, int n_bins, const double2* emean, const uint32_t* nacc,
                                const uint32_t* nprop, int n_chains, double* scratch, EpochStatsDev* out,
                                cudaStream_t st) {
    if (n_bins < 1 || n_bins > kMaxBins || N % n_bins) return cudaErrorInvalidValue;
    energy_stats<<<n_bins, 256, 0, st>>>(E, N, n_bins, emean, nacc, nprop, n_chains, scratch, out);
    return cudaGetLastError();
}

int gram_splits(int N, int P) {
    const int nt = (P + GT - 1) / GT;
    const int tiles = nt * (nt + 1) / 2;
    int ks = (2 * 148 + tiles - 1) / tiles;
    if (ks > 64) ks = 64;
    if (ks > N / GK) ks = N / GK > 0 ? N / GK : 1;
    return ks < 1 ? 1 : ks;
}

cudaError_t launch_gram_fp64(const void* O, int fp64, const double2* d, int N, int P, int nks, double2* part,
                             double2* S, cudaStream_t st) {
    const int nt = (P + GT - 1) / GT;
    dim3 grid(nt * (nt + 1) / 2, nks);
    if (fp64)
        gram_fp64<double2><<<grid, 256, 0, st>>>((const double2*)O, d, N, P, nt, part);
    else
        gram_fp64<float2><<<grid, 256, 0, st>>>((const float2*)O, d, N, P, nt, part);
    gram_finalize<<<296, 256, 0, st>>>(part, nks, N, P, S);
    return cudaGetLastError();
}

cudaError_t launch_schedule(ScheduleDev* s, cudaStream_t st) {
    schedule_step<<<1, 32, 0, st>>>(s, 0);
    return cudaGetLastError();
}

cudaError_t launch_schedule_regs(ScheduleDev* s, cudaStream_t st) {
    schedule_step<<<1, 32, 0, st>>>(s, 1);
    return cudaGetLastError();
}

cudaError_t launch_regularize(const double2* S, int P, int n_neural, int N, const ScheduleDev* sch, double* diag,
                              double2* Sreg, double* max_diag, cudaStream_t st, int direct, const double* vfac) {
    const int blocks = (int)std::max<long>(1, std::min<long>(296, ((long)P * P + 1023) / 1024));
    regularize<<<blocks, 1024, 0, st>>>(S, P, n_neural, N, sch, diag, Sreg, max_diag, direct, vfac);
    return cudaGetLastError();
}

bool cg_cluster_fits(int P) {
    const int rp = (P + kClusterCta - 1) / kClusterCta;
    return ((size_t)rp * P + 2 * (size_t)P + 2 * (size_t)rp) * sizeof(double2) <= 200 * 1024;
}

cudaError_t launch_cg(const double2* A, const double2* b, double2* x, int P, int max_it, double rtol, CgResultDev* res,
                      cudaStream_t st) {
    const int rp = (P + kClusterCta - 1) / kClusterCta;
    const size_t csm = ((size_t)rp * P + 2 * (size_t)P + 2 * (size_t)rp) * sizeof(double2);
    if (csm <= 200 * 1024) {
        cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(cg_cluster), (int)csm);
        if (e != cudaSuccess) return e;
        cg_cluster<<<kClusterCta, 256, csm, st>>>(A, b, x, P, max_it, rtol, res);
        return cudaGetLastError();
    }
    const size_t packed = (packed_size(P) + 4 * (size_t)P) * sizeof(double2);
    if (packed <= 200 * 1024) {
        cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(cg_packed), (int)packed);
        if (e != cudaSuccess) return e;
        cg_packed<<<1, 1024, packed, st>>>(A, b, x, P, max_it, rtol, res);
        return cudaGetLastError();
    }
    const int smem = 3 * P * (int)sizeof(double2);
    cudaError_t e = ensure_dynamic_smem(reinterpret_cast<const void*>(cg_dense), smem);
    if (e != cudaSuccess) return e;
    cg_dense<<<1, 1024, smem, st>>>(A, b, x, P, max_it, rtol, res);
    return cudaGetLastError();
}

cudaError_t launch_update(double2* params, double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                          cudaStream_t st) {
    sr_update<<<1, 1024, 0, st>>>(params, x, P, sch, res, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_update(double2* params, double2* x, int P, const ScheduleDev* sch, CgResultDev* res,
                          PluginDev* plug, cudaStream_t st) {
    sr_update<<<1, 1024, 0, st>>>(params, x, P, sch, res, plug);
    return cudaGetLastError();
}

__global__ void sgd_direction(const double2* F, double2* x, int P, double real_factor, CgResultDev* res) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
        const double2 f = F[i];
        x[i] = make_double2(f.x / real_factor, f.y);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        res->iterations = 0;
        res->residual = 0;
        res->status = 0;
    }
}

cudaError_t launch_sgd_direction(const double2* F, double2* x, int P, double real_factor, CgResultDev* res,
                                 cudaStream_t st) {
    sgd_direction<<<(P + 255) / 256, 256, 0, st>>>(F, x, P, real_factor, res);
    return cudaGetLastError();
}

cudaError_t launch_unpack(const double2* params, int n, int n_vb, int nh, double2* vb, double2* hb, double2* W64,
                          float2* W32, cudaStream_t st) {
    unpack_weights<<<148, 256, 0, st>>>(params, n, n_vb, nh, vb, hb, W64, W32);
    return cudaGetLastError();
}

}  // namespace rbmnqs
