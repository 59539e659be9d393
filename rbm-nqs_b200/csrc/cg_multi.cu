// cg_multi.cu -- matrix-free SR conjugate gradients of several independent
// systems in one cooperative persistent launch (cg_solver.cpp:260-334, cg1
// semantics, with the operator of cg_solver.cpp aprod):
//
//   A b = (1/N) O^H (O b) - conj(d) (d . b) + f o b,
//   f_p = diag_p (r1 (+ rd for non-neural p)) + r2 max(diag),
//
// warm start x0, stop at ||r||^2 < rtol or after max_it iterations, each
// system on its own.  Every system of the launch advances in lockstep and
// the systems share the grid barriers: three per iteration.
//
//   A  rows:    v = O b (8 rows per unit, the block's 8 warps split the
//               columns, each lane two adjacent columns per load, slice sums
//               added in slice order), and d . b per 128-column tile;
//   B  columns: Ap = O^H v / N - conj(d) (d . b) + f o b per 128-column
//               tile (each thread a column pair), p^H A p per tile;
//   C  update:  x += alpha p, r -= alpha Ap per tile, ||r||^2 per tile.
//
// b is the iteration's search direction p = r + beta p_prev, formed on the
// fly where it is read (double-buffered p: phase B of the tile's owner
// stores it for phase C and the next iteration).  Units are handed to blocks
// as contiguous ranges of equal cost; every per-system sum is formed in a
// fixed order (slices in order, then tiles in order, one warp per system),
// so a system's result depends neither on the grid nor on the other systems
// of the launch.  Barriers are bounded (coop.cuh): a timeout marks every
// system's result with status -2 and the kernel returns.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "coop.cuh"
#include "sr.cuh"

namespace rbmnqs {
namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kRows = 8;     // rows per phase-A unit (each b element read serves 8 rows)
constexpr int kTile = 128;   // columns per phase-B/C tile: 64 column pairs x 4 row groups
constexpr int kPairs = kTile / 2;
constexpr int kGroups = kThreads / kPairs;
// Streaming ring: O (and the b inputs of phase A, v of phase B) are copied
// into shared memory with cp.async, kStages chunks deep, kAhead in flight
// while one is consumed; one 512-thread block per SM.
constexpr int kStages = 4;
constexpr int kAhead = kStages - 1;
constexpr int kStageO = 32 * 1024;                    // O bytes per chunk
constexpr int kStageBytes = kStageO + 16 * 1024;      // + phase A: r and p_prev (or x) of the chunk's columns
constexpr int kRingBytes = kStages * kStageBytes;

__device__ __forceinline__ void cp16(uint32_t s, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(g) : "memory");
}
// 8-byte copies of O only (read-only during the kernel; cached in L1)
__device__ __forceinline__ void cp8(uint32_t s, const void* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }

template <typename T> __device__ __forceinline__ T ld_l2(const T* p) { return __ldcg(p); }

// per-system scalars every block carries (the same values on every block)
struct SysState {
    double rsold, beta, db_x, db_y, ax, ay, rs;
    int itn, done, pad;
};

// [lo, hi) of the units whose start cost lies in this block's share of the
// total cost; cost0 = first unit's start, unit_cost = per-unit cost
__device__ __forceinline__ void owned(long long c0, long long c1, long long cost0, long long unit_cost, int units,
                                      int& lo, int& hi) {
    auto first_at = [&](long long c) -> long long {  // first unit whose start >= c
        if (c <= cost0) return 0;
        return (c - cost0 + unit_cost - 1) / unit_cost;
    };
    lo = (int)std::min<long long>(first_at(c0), units);
    hi = (int)std::min<long long>(first_at(c1), units);
}

// conj-free complex multiply-accumulate a += o b, and a += conj(o) b
__device__ __forceinline__ void cmac(double& ax, double& ay, double2 o, double2 b) {
    ax = fma(o.x, b.x, fma(-o.y, b.y, ax));
    ay = fma(o.x, b.y, fma(o.y, b.x, ay));
}
__device__ __forceinline__ void cmacc(double& ax, double& ay, double2 o, double2 b) {
    ax = fma(o.x, b.x, fma(o.y, b.y, ax));
    ay = fma(o.x, b.y, fma(-o.y, b.x, ay));
}

template <typename TO>
__global__ void __launch_bounds__(kThreads) cg_multi_kernel(const CgMultiProb* __restrict__ probs, int nprob,
                                                            CgMultiScratch s) {
    __shared__ CgMultiProb pr[kCgMultiMax];
    __shared__ SysState ss[kCgMultiMax];
    __shared__ double2 rowred[kWarps][kRows];
    __shared__ double2 colred[2][kThreads];
    __shared__ double2 tred[kWarps];
    __shared__ double tred_d[kWarps];
    __shared__ int any_active;
    extern __shared__ __align__(16) unsigned char ring[];
    const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
    constexpr int ES = (int)sizeof(TO);
    constexpr int CW = kStageO / (kRows * ES);   // phase A: columns per chunk (512 FP32, 256 FP64)
    constexpr int RB = kStageO / (kTile * ES);   // phase B: rows per chunk (32 FP32, 16 FP64)
    const int G = gridDim.x, blk = blockIdx.x;
    for (int i = tid; i < nprob; i += kThreads) pr[i] = probs[i];
    if (tid < nprob) ss[tid] = SysState{};
    __syncthreads();
    // this block's contiguous share of the row units and of the tiles
    const long long rc0 = s.row_cost * blk / G, rc1 = s.row_cost * (blk + 1) / G;
    const long long tc0 = s.tile_cost * blk / G, tc1 = s.tile_cost * (blk + 1) / G;

    // b_q of system i: x (init) or p = r + beta p_prev, p_prev in the buffer
    // of the other parity (iteration k stores its p in buffer k & 1)
    auto bval = [&](const CgMultiProb& p, const SysState& st, int q, bool init, int par) -> double2 {
        if (init) return ld_l2(p.x + q);
        const double2 r = ld_l2(p.r + q);
        if (st.beta == 0.0) return r;
        const double2 pp = ld_l2((par ? p.p0 : p.p1) + q);
        return make_double2(fma(st.beta, pp.x, r.x), fma(st.beta, pp.y, r.y));
    };
    // sum of the per-warp values of warps 0 .. nw-1 in warp order (thread 0)
    auto block_tile_sum2 = [&](double2 v, int nw) -> double2 {
        if (wib < nw) {
            v.x = warp_sum(v.x);
            v.y = warp_sum(v.y);
            if (lane == 0) tred[wib] = v;
        }
        __syncthreads();
        double2 t = tred[0];
        for (int w = 1; w < nw; w++) t = make_double2(t.x + tred[w].x, t.y + tred[w].y);
        return t;
    };
    auto block_tile_sum1 = [&](double v, int nw) -> double {
        if (wib < nw) {
            v = warp_sum(v);
            if (lane == 0) tred_d[wib] = v;
        }
        __syncthreads();
        double t = tred_d[0];
        for (int w = 1; w < nw; w++) t += tred_d[w];
        return t;
    };

    // phase A: O b of the owned row units, d . b of the owned tiles.  A unit
    // (8 rows) streams through the ring in chunks of CW columns: O rows and
    // the b inputs (x, or r and p_prev) of the chunk's columns; thread t
    // takes the columns t, t + 512, ... of each chunk and keeps 8 row
    // partials, summed over the block in a fixed order at the unit's end.
    auto phase_a = [&](bool init, int par) {
        for (int i = 0; i < nprob; i++) {
            const CgMultiProb& p = pr[i];
            const SysState st = ss[i];
            if (st.done) continue;
            const int P = p.P, N = p.N;
            const bool vec = (P * ES) % 16 == 0;
            const bool two = !init && st.beta != 0.0;
            const double2* b1 = init ? p.x : p.r;
            const double2* b2 = par ? p.p0 : p.p1;
            const TO* O = reinterpret_cast<const TO*>(p.O);
            int u0, u1;
            owned(rc0, rc1, p.row_cost0, (long long)P, (N + kRows - 1) / kRows, u0, u1);
            const int nch = (P + CW - 1) / CW;
            for (int u = u0; u < u1; u++) {
                const int n0 = u * kRows;
                const int nr = min(kRows, N - n0);
                auto issue = [&](int k) {
                    if (k < nch) {
                        unsigned char* sg = ring + (k % kStages) * kStageBytes;
                        const int cs = k * CW, cw = min(CW, P - cs);
                        if (vec && cw == CW) {
                            // full chunk: SEGS 16-byte segments per row, RPP rows per pass
                            constexpr int SEGS = CW * ES / 16, RPP = kThreads / SEGS;
                            const int h = tid % SEGS, r0 = tid / SEGS;
                            const char* src = reinterpret_cast<const char*>(O + (size_t)(n0 + r0) * P + cs) + 16 * h;
                            const size_t rstep = (size_t)RPP * P * ES;
                            uint32_t dst = saddr(sg + r0 * (CW * ES) + 16 * h);
                            for (int r = r0; r < nr; r += RPP) {
                                cp16(dst, src);
                                src += rstep;
                                dst += RPP * (CW * ES);
                            }
                        } else if (vec) {
                            const int segs = cw * ES / 16;
                            for (int r = 0; r < nr; r++) {
                                const char* src = reinterpret_cast<const char*>(O + (size_t)(n0 + r) * P + cs);
                                for (int g = tid; g < segs; g += kThreads)
                                    cp16(saddr(sg + r * (CW * ES) + 16 * g), src + 16 * g);
                            }
                        } else {
                            for (int r = 0; r < nr; r++) {
                                const TO* src = O + (size_t)(n0 + r) * P + cs;
                                for (int c = tid; c < cw; c += kThreads) cp8(saddr(sg + r * (CW * ES) + 8 * c), src + c);
                            }
                        }
                        double2* bs = reinterpret_cast<double2*>(sg + kStageO);
                        for (int c = tid; c < cw; c += kThreads) {
                            cp16(saddr(bs + c), b1 + cs + c);
                            if (two) cp16(saddr(bs + CW + c), b2 + cs + c);
                        }
                    }
                    cp_commit();
                };
                double ax[kRows], ay[kRows];
#pragma unroll
                for (int r = 0; r < kRows; r++) ax[r] = ay[r] = 0.0;
                for (int k = 0; k < kAhead; k++) issue(k);
                for (int k = 0; k < nch; k++) {
                    // chunk k landed (this thread's copies), then everyone's
                    // copies are visible and everyone is done with chunk k - 1,
                    // whose stage takes chunk k + kAhead
                    cp_wait<kAhead - 1>();
                    __syncthreads();
                    issue(k + kAhead);
                    const unsigned char* sg = ring + (k % kStages) * kStageBytes;
                    const TO* Os = reinterpret_cast<const TO*>(sg);
                    const double2* bs = reinterpret_cast<const double2*>(sg + kStageO);
                    const int cw = min(CW, P - k * CW);
                    for (int c = tid; c < cw; c += kThreads) {
                        double2 b = bs[c];
                        if (two) {
                            const double2 pp = bs[CW + c];
                            b = make_double2(fma(st.beta, pp.x, b.x), fma(st.beta, pp.y, b.y));
                        }
#pragma unroll
                        for (int r = 0; r < kRows; r++)
                            if (r < nr) cmac(ax[r], ay[r], to_d2(Os[r * CW + c]), b);
                    }
                }
#pragma unroll
                for (int r = 0; r < kRows; r++) {
                    const double sx = warp_sum(ax[r]), sy = warp_sum(ay[r]);
                    if (lane == 0) rowred[wib][r] = make_double2(sx, sy);
                }
                __syncthreads();
                if (tid < nr) {
                    double2 t = rowred[0][tid];
                    for (int j = 1; j < kWarps; j++) t = make_double2(t.x + rowred[j][tid].x, t.y + rowred[j][tid].y);
                    p.v[n0 + tid] = t;
                }
                __syncthreads();
            }
            // d . b per owned tile: threads 0..127 one column each
            int t0, t1;
            owned(tc0, tc1, p.tile_cost0, (long long)N, (P + kTile - 1) / kTile, t0, t1);
            for (int t = t0; t < t1; t++) {
                const int q = t * kTile + tid;
                double2 db = make_double2(0, 0);
                if (tid < kTile && q < P) {
                    const double2 dq = p.d[q], v = bval(p, st, q, init, par);
                    db.x = dq.x * v.x - dq.y * v.y;
                    db.y = dq.x * v.y + dq.y * v.x;
                }
                const double2 tot = block_tile_sum2(db, kTile / 32);
                if (tid == 0) s.tdb[p.tile0 + t] = tot;
                __syncthreads();
            }
        }
    };

    // per-system totals of tile partials, one warp per system, tiles in order
    auto reduce2 = [&](const double2* part, int which) {
        for (int i = wib; i < nprob; i += kWarps) {
            const CgMultiProb& p = pr[i];
            if (ss[i].done) continue;
            const int nt = (p.P + kTile - 1) / kTile;
            double sx = 0, sy = 0;
            for (int t = lane; t < nt; t += 32) {
                const double2 v = ld_l2(part + p.tile0 + t);
                sx += v.x;
                sy += v.y;
            }
            sx = warp_sum(sx);
            sy = warp_sum(sy);
            if (lane == 0) {
                if (which == 0) {
                    ss[i].db_x = sx;
                    ss[i].db_y = sy;
                } else {
                    ss[i].ax = sx;
                    ss[i].ay = sy;
                }
            }
        }
        __syncthreads();
    };
    auto reduce1 = [&](const double* part) {
        for (int i = wib; i < nprob; i += kWarps) {
            const CgMultiProb& p = pr[i];
            if (ss[i].done) continue;
            const int nt = (p.P + kTile - 1) / kTile;
            double sx = 0;
            for (int t = lane; t < nt; t += 32) sx += ld_l2(part + p.tile0 + t);
            sx = warp_sum(sx);
            if (lane == 0) ss[i].rs = sx;
        }
        __syncthreads();
    };

    // phase B over the owned tiles: Ap (init: r = F - Ap and ||r||^2 per
    // tile; else p stored and p^H A p per tile); thread (c, rg) takes the
    // column pair c of the tile over the rows rg, rg + 4, ...
    auto phase_b = [&](bool init, int par) {
        const int c = tid % kPairs, rg = tid / kPairs;
        for (int i = 0; i < nprob; i++) {
            const CgMultiProb& p = pr[i];
            const SysState st = ss[i];
            if (st.done) continue;
            const int P = p.P, N = p.N;
            const TO* O = reinterpret_cast<const TO*>(p.O);
            const double r1 = p.sch ? p.sch->value[1] : 0.0, r2 = p.sch ? p.sch->value[2] : 0.0,
                         rd = p.sch ? p.sch->value[3] : 0.0;
            const double mxd = p.max_diag ? *p.max_diag : 0.0;
            int t0, t1;
            owned(tc0, tc1, p.tile_cost0, (long long)N, (P + kTile - 1) / kTile, t0, t1);
            const bool vec = (P * ES) % 16 == 0;
            const int nch = (N + RB - 1) / RB;
            for (int t = t0; t < t1; t++) {
                const int qs = t * kTile, tw = min(kTile, P - qs);
                auto issue = [&](int k) {
                    if (k < nch) {
                        unsigned char* sg = ring + (k % kStages) * kStageBytes;
                        const int ns = k * RB, rows = min(RB, N - ns);
                        if (vec && tw == kTile) {
                            // full tile: SEGS 16-byte segments per row, RPP rows per pass
                            constexpr int SEGS = kTile * ES / 16, RPP = kThreads / SEGS;
                            const int h = tid % SEGS, r0 = tid / SEGS;
                            const char* src = reinterpret_cast<const char*>(O + (size_t)(ns + r0) * P + qs) + 16 * h;
                            const size_t rstep = (size_t)RPP * P * ES;
                            uint32_t dst = saddr(sg + r0 * (kTile * ES) + 16 * h);
                            for (int r = r0; r < rows; r += RPP) {
                                cp16(dst, src);
                                src += rstep;
                                dst += RPP * (kTile * ES);
                            }
                        } else if (vec) {
                            const int segs = tw * ES / 16;  // per row
                            for (int g = tid; g < rows * segs; g += kThreads) {
                                const int r = g / segs, h = g - r * segs;
                                cp16(saddr(sg + r * (kTile * ES) + 16 * h),
                                     reinterpret_cast<const char*>(O + (size_t)(ns + r) * P + qs) + 16 * h);
                            }
                        } else {
                            for (int g = tid; g < rows * tw; g += kThreads) {
                                const int r = g / tw, h = g - r * tw;
                                cp8(saddr(sg + r * (kTile * ES) + 8 * h), O + (size_t)(ns + r) * P + qs + h);
                            }
                        }
                        double2* vs = reinterpret_cast<double2*>(sg + kStageO);
                        for (int r = tid; r < rows; r += kThreads) cp16(saddr(vs + r), p.v + ns + r);
                    }
                    cp_commit();
                };
                double a0x = 0, a0y = 0, a1x = 0, a1y = 0;
                for (int k = 0; k < kAhead; k++) issue(k);
                for (int k = 0; k < nch; k++) {
                    cp_wait<kAhead - 1>();  // as in phase A: one barrier per chunk
                    __syncthreads();
                    issue(k + kAhead);
                    const unsigned char* sg = ring + (k % kStages) * kStageBytes;
                    const TO* Os = reinterpret_cast<const TO*>(sg);
                    const double2* vs = reinterpret_cast<const double2*>(sg + kStageO);
                    const int rows = min(RB, N - k * RB);
                    if (2 * c + 1 < tw) {
                        for (int rr = rg; rr < rows; rr += kGroups) {
                            const double2 v = vs[rr];
                            double2 o0, o1;
                            if constexpr (ES == 8) {  // the column pair in one 16-byte load
                                const float4 w = *reinterpret_cast<const float4*>(Os + rr * kTile + 2 * c);
                                o0 = make_double2(w.x, w.y);
                                o1 = make_double2(w.z, w.w);
                            } else {
                                o0 = to_d2(Os[rr * kTile + 2 * c]);
                                o1 = to_d2(Os[rr * kTile + 2 * c + 1]);
                            }
                            cmacc(a0x, a0y, o0, v);
                            cmacc(a1x, a1y, o1, v);
                        }
                    } else if (2 * c < tw) {
                        for (int rr = rg; rr < rows; rr += kGroups) cmacc(a0x, a0y, to_d2(Os[rr * kTile + 2 * c]), vs[rr]);
                    }
                }
                colred[0][tid] = make_double2(a0x, a0y);
                colred[1][tid] = make_double2(a1x, a1y);
                __syncthreads();
                // threads 0..127: one column each (column q0 + tid of the tile)
                double2 part = make_double2(0, 0);
                double rpart = 0;
                const int qc = t * kTile + tid;
                if (tid < kTile && qc < P) {
                    const int cc = tid >> 1, h = tid & 1;
                    double sx = 0, sy = 0;
                    for (int g = 0; g < kGroups; g++) {
                        sx += colred[h][g * kPairs + cc].x;
                        sy += colred[h][g * kPairs + cc].y;
                    }
                    const double2 dq = p.d[qc], bq = bval(p, st, qc, init, par);
                    const double f = p.diag[qc] * (qc < p.n_neural ? r1 : r1 + rd) + mxd * r2;
                    double2 a;
                    a.x = f * bq.x + sx / p.norm - (dq.x * st.db_x + dq.y * st.db_y);
                    a.y = f * bq.y + sy / p.norm - (dq.x * st.db_y - dq.y * st.db_x);
                    if (init) {
                        const double2 fq = p.F[qc];
                        const double2 rq = make_double2(fq.x - a.x, fq.y - a.y);
                        p.r[qc] = rq;
                        rpart = rq.x * rq.x + rq.y * rq.y;
                    } else {
                        p.Ap[qc] = a;
                        (par ? p.p1 : p.p0)[qc] = bq;
                        part.x = bq.x * a.x + bq.y * a.y;
                        part.y = bq.x * a.y - bq.y * a.x;
                    }
                }
                if (init) {
                    const double tot = block_tile_sum1(rpart, kTile / 32);
                    if (tid == 0) s.trs[p.tile0 + t] = tot;
                } else {
                    const double2 tot = block_tile_sum2(part, kTile / 32);
                    if (tid == 0) s.tpap[p.tile0 + t] = tot;
                }
                __syncthreads();
            }
        }
    };

    // phase C over the owned tiles: x += alpha p, r -= alpha Ap, ||r||^2 per tile
    auto phase_c = [&](int par) {
        for (int i = 0; i < nprob; i++) {
            const CgMultiProb& p = pr[i];
            const SysState st = ss[i];
            if (st.done) continue;
            // alpha = rsold / (p^H A p)
            const double den = st.ax * st.ax + st.ay * st.ay;
            const double al_x = st.rsold * st.ax / den, al_y = -st.rsold * st.ay / den;
            int t0, t1;
            owned(tc0, tc1, p.tile_cost0, (long long)p.N, (p.P + kTile - 1) / kTile, t0, t1);
            for (int t = t0; t < t1; t++) {
                const int q = t * kTile + tid;
                double rl = 0;
                if (tid < kTile && q < p.P) {
                    const double2 pq = ld_l2((par ? p.p1 : p.p0) + q), aq = ld_l2(p.Ap + q);
                    double2 xq = ld_l2(p.x + q), rq = ld_l2(p.r + q);
                    xq.x += al_x * pq.x - al_y * pq.y;
                    xq.y += al_x * pq.y + al_y * pq.x;
                    rq.x -= al_x * aq.x - al_y * aq.y;
                    rq.y -= al_x * aq.y + al_y * aq.x;
                    p.x[q] = xq;
                    p.r[q] = rq;
                    rl = rq.x * rq.x + rq.y * rq.y;
                }
                const double tot = block_tile_sum1(rl, kTile / 32);
                if (tid == 0) s.trs[p.tile0 + t] = tot;
                __syncthreads();
            }
        }
    };

    bool ok = true;
    // r = F - A x0, p = r
    phase_a(true, 0);
    ok = grid_barrier(s.sync, G);
    if (ok) {
        reduce2(s.tdb, 0);
        phase_b(true, 0);
        ok = grid_barrier(s.sync, G);
    }
    if (ok) {
        reduce1(s.trs);
        if (tid < nprob) {
            SysState& st = ss[tid];
            st.rsold = st.rs;
            st.beta = 0.0;
            st.itn = 0;
            st.done = pr[tid].max_it <= 0;
        }
        __syncthreads();
    }
    int par = 0;
    while (ok) {
        if (tid == 0) {
            int a = 0;
            for (int i = 0; i < nprob; i++) a |= !ss[i].done;
            any_active = a;
        }
        __syncthreads();
        if (!any_active) break;
        phase_a(false, par);
        if (!(ok = grid_barrier(s.sync, G))) break;
        reduce2(s.tdb, 0);
        phase_b(false, par);
        if (!(ok = grid_barrier(s.sync, G))) break;
        reduce2(s.tpap, 1);
        phase_c(par);
        if (!(ok = grid_barrier(s.sync, G))) break;
        reduce1(s.trs);
        if (tid < nprob) {
            SysState& st = ss[tid];
            if (!st.done) {
                if (st.rs < pr[tid].rtol) {
                    st.done = 1;  // cg1: stop before the direction update, itn not advanced
                } else {
                    st.beta = st.rs / st.rsold;
                    st.rsold = st.rs;
                    st.itn++;
                    if (st.itn >= pr[tid].max_it) st.done = 1;
                }
            }
        }
        __syncthreads();
        par ^= 1;
    }
    if (blk == 0 && tid < nprob) {
        CgResultDev* res = pr[tid].res;
        res->status = ok ? 0 : -2;
        res->istop = 0;
        res->qlp_iterations = 0;
        res->acond = 0;
        res->iterations = ss[tid].itn;
        res->residual = ss[tid].rs;
    }
}

}  // namespace

int cg_multi_units(CgMultiProb* probs, int nprob, long long* row_cost, long long* tile_cost) {
    long long rc = 0, tc = 0;
    int tiles = 0;
    for (int i = 0; i < nprob; i++) {
        CgMultiProb& p = probs[i];
        p.row_cost0 = rc;
        p.tile_cost0 = tc;
        p.tile0 = tiles;
        const int units = (p.N + kRows - 1) / kRows, nt = (p.P + kTile - 1) / kTile;
        rc += (long long)units * p.P;
        tc += (long long)nt * p.N;
        tiles += nt;
    }
    *row_cost = rc;
    *tile_cost = tc;
    return tiles;
}

cudaError_t cg_multi_blocks(int* blocks) {
    int dev = 0, sms = 148, coop = 0, b32 = 0, b64 = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return cudaErrorNotSupported;
    const void* f32 = reinterpret_cast<const void*>(cg_multi_kernel<float2>);
    const void* f64 = reinterpret_cast<const void*>(cg_multi_kernel<double2>);
    if ((e = ensure_dynamic_smem(f32, kRingBytes)) != cudaSuccess) return e;
    if ((e = ensure_dynamic_smem(f64, kRingBytes)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b32, cg_multi_kernel<float2>, kThreads, kRingBytes)) !=
        cudaSuccess)
        return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b64, cg_multi_kernel<double2>, kThreads, kRingBytes)) !=
        cudaSuccess)
        return e;
    const int per_sm = std::min(b32, b64);
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    *blocks = sms * per_sm;  // one block per SM (the ring takes most of the shared memory)
    return cudaSuccess;
}

cudaError_t launch_cg_multi(const CgMultiProb* probs_dev, int nprob, int fp64, const CgMultiScratch& s, int blocks,
                            cudaStream_t st) {
    if (nprob < 1 || nprob > kCgMultiMax || blocks < 1) return cudaErrorInvalidValue;
    cudaError_t e = launch_init_sync(s.sync, st);
    if (e != cudaSuccess) return e;
    CgMultiScratch sc = s;
    const CgMultiProb* p = probs_dev;
    int np = nprob;
    void* args[] = {&p, &np, &sc};
    const void* fn = fp64 ? reinterpret_cast<const void*>(cg_multi_kernel<double2>)
                          : reinterpret_cast<const void*>(cg_multi_kernel<float2>);
    if ((e = ensure_dynamic_smem(fn, kRingBytes)) != cudaSuccess) return e;
    return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kThreads), args, kRingBytes, st);
}

}  // namespace rbmnqs
