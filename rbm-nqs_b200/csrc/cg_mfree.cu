// cg_mfree.cu -- matrix-free SR conjugate gradients for parameter counts
// whose P x P matrix S is not formed (cg_solver.cpp:260-334 with the
// operator of minresqlp_adapter.cpp / cg_solver.cpp aprod):
//
//   A b = (1/N) O^H (O b) - conj(d) (d . b) + f o b,
//   f_p = diag_p (r1 (+ rd for non-neural p)) + r2 max(diag),
//
// cg1 semantics (warm start x0, stop at ||r||^2 < rtol or max_it).  One
// cooperative persistent kernel runs the whole solve; per iteration it
// streams O twice (rows for O b, columns for O^H v) and meets at five grid
// barriers.  The barriers are a counter + generation pair with bounded
// spins: a block that waits too long records an error and the solve returns
// (status RBMNQS_ERR_CUDA) instead of hanging.  Reductions are summed in a
// fixed order, so results are deterministic.
#include <cooperative_groups.h>

#include <algorithm>

#include "common.cuh"
#include "coop.cuh"
#include "sr.cuh"

namespace rbmnqs {
namespace {

constexpr int kThreads = 256;
constexpr int kColTile = 64;  // columns per block in the O^H v pass (4 row groups)

__device__ __forceinline__ double2 zld(const float2* O, size_t i) {
    const float2 v = __ldg(O + i);
    return make_double2(v.x, v.y);
}
__device__ __forceinline__ double2 zld(const double2* O, size_t i) { return __ldg(O + i); }

// Data written by other blocks of the same launch is read through L2
// (ld.global.cg): the SMs' L1 caches are not coherent with each other.
template <typename T> __device__ __forceinline__ T cg_ld(const T* p) { return __ldcg(p); }

template <typename T> __device__ T bsum(T v, T* red);
template <> __device__ double bsum<double>(double v, double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double r = red[0];
    for (int i = 1; i < nw; i++) r += red[i];
    return r;
}
template <> __device__ double2 bsum<double2>(double2 v, double2* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v.x = warp_sum(v.x);
    v.y = warp_sum(v.y);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double2 r = red[0];
    for (int i = 1; i < nw; i++) r = make_double2(r.x + red[i].x, r.y + red[i].y);
    return r;
}

// Sum of the per-block partials: thread t adds entries t, t + 256, ... and the
// block reduces in a fixed order, so every block gets the same value (and the
// loads are issued in parallel rather than as one dependent chain).
// Stable reflection [c s; s -c] (a, b)^T = (r, 0)^T for real a, b with c >= 0
// (SYMORTHO of MINRES-QLP, zminresqlpModule.f90): the larger of |a|, |b|
// divides, so nothing overflows or cancels.
__device__ __forceinline__ void symortho(double a, double b, double& c, double& s, double& r) {
    const double aa = fabs(a), ab = fabs(b), rmin = 2.2250738585072014e-308;
    const double sg = (a > 0) == (b > 0) ? 1.0 : -1.0;
    if (ab <= rmin) {
        c = 1, s = 0, r = a;
    } else if (aa <= rmin) {
        c = 0, s = 1, r = b;
    } else if (ab > aa) {
        const double t = aa / ab, cc = 1.0 / sqrt(1.0 + t * t);
        s = cc * sg;
        c = cc * t;
        r = b / s;
    } else {
        const double t = ab / aa, cc = 1.0 / sqrt(1.0 + t * t);
        c = cc;
        s = cc * t * sg;
        r = a / cc;
    }
}

__device__ __forceinline__ double sum_parts(const double* p, int G, double* red) {
    double s = 0;
    for (int i = threadIdx.x; i < G; i += blockDim.x) s += cg_ld(p + i);
    return bsum(s, red);
}
__device__ __forceinline__ double2 sum_parts(const double2* p, int G, double2* red) {
    double2 s = make_double2(0, 0);
    for (int i = threadIdx.x; i < G; i += blockDim.x) {
        const double2 v = cg_ld(p + i);
        s = make_double2(s.x + v.x, s.y + v.y);
    }
    return bsum(s, red);
}

template <typename TO>
__global__ void __launch_bounds__(kThreads) cg_mfree_kernel(const TO* __restrict__ O, const double2* __restrict__ d,
                                                            double norm, int N, int P, int n_neural,
                                                            const double2* __restrict__ F, double2* x,
                                                            const double* __restrict__ diag, const double* max_diag,
                                                            const ScheduleDev* sch, double r1_, double r2_,
                                                            double rd_, int max_it, double rtol, MfreeWork w,
                                                            CgResultDev* res) {
    __shared__ double redd[kThreads / 32];
    __shared__ double2 redz[kThreads / 32];
    __shared__ double2 colred[kThreads];
    const int tid = threadIdx.x, lane = tid & 31;
    const int G = gridDim.x, blk = blockIdx.x;
    const int gw = blk * (kThreads / 32) + (tid >> 5), nwarps = G * (kThreads / 32);
    const int gt = blk * kThreads + tid, nthreads = G * kThreads;
    const double r1 = sch ? sch->value[1] : r1_, r2 = sch ? sch->value[2] : r2_, rd = sch ? sch->value[3] : rd_;
    const double mxd = max_diag ? *max_diag : 0.0;
    if (blk == 0 && tid == 0) {
        res->status = 0;
        res->istop = 0;
        res->qlp_iterations = 0;
        res->acond = 0;
    }

    // A b into Ap (b = x at the start, p afterwards); returns false on a
    // barrier timeout.  With want_pap, also leaves sum_q conj(b_q) Ap_q.
    auto aprod = [&](const double2* b, bool want_pap, double2* pap) -> bool {
        if (w.S) {
            // formed, regularised S: Ap = S b, one warp per row
            double2 pp = make_double2(0, 0);
            for (int r = gw; r < P; r += nwarps) {
                const double2* Sr = w.S + (size_t)r * P;
                double ax = 0, ay = 0;
                int q = lane;
                for (; q + 96 < P; q += 128) {
                    double2 a[4], v[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        a[u] = __ldg(Sr + q + 32 * u);
                        v[u] = cg_ld(b + q + 32 * u);
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        ax = fma(a[u].x, v[u].x, fma(-a[u].y, v[u].y, ax));
                        ay = fma(a[u].x, v[u].y, fma(a[u].y, v[u].x, ay));
                    }
                }
                for (; q < P; q += 32) {
                    const double2 a = __ldg(Sr + q), v = cg_ld(b + q);
                    ax = fma(a.x, v.x, fma(-a.y, v.y, ax));
                    ay = fma(a.x, v.y, fma(a.y, v.x, ay));
                }
                ax = warp_sum(ax);
                ay = warp_sum(ay);
                if (lane == 0) {
                    w.Ap[r] = make_double2(ax, ay);
                    if (want_pap) {
                        const double2 br = cg_ld(b + r);
                        pp.x += br.x * ax + br.y * ay;
                        pp.y += br.x * ay - br.y * ax;
                    }
                }
            }
            if (want_pap) {
                pp = bsum(pp, redz);
                if (tid == 0) w.zpart[blk] = pp;
            }
            if (!grid_barrier(w.sync, G)) return false;
            if (want_pap) *pap = sum_parts(w.zpart, G, redz);
            return true;
        }
        // phase A: O b.  Block blk owns rows blk, blk + G, ...; its 8 warps
        // split the columns into 8 slices and walk 4 rows at a time, so each
        // b element read from L2 serves 4 rows.  Partial dots per (slice, row).
        {
            const int wib = tid >> 5, nwb = kThreads / 32;
            const int q0 = (int)((long)P * wib / nwb), q1 = (int)((long)P * (wib + 1) / nwb);
            for (int n0 = blk; n0 < N; n0 += 4 * G) {
                int nr[4];
                bool val[4];
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    nr[r] = n0 + r * G;
                    val[r] = nr[r] < N;
                }
                double ax[4] = {0, 0, 0, 0}, ay[4] = {0, 0, 0, 0};
                for (int q = q0 + lane; q < q1; q += 32) {
                    const double2 v = cg_ld(b + q);
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        if (!val[r]) continue;
                        const double2 o = zld(O, (size_t)nr[r] * P + q);
                        ax[r] = fma(o.x, v.x, fma(-o.y, v.y, ax[r]));
                        ay[r] = fma(o.x, v.y, fma(o.y, v.x, ay[r]));
                    }
                }
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    const double sx = warp_sum(ax[r]), sy = warp_sum(ay[r]);
                    if (lane == 0 && val[r]) w.partA[(size_t)wib * N + nr[r]] = make_double2(sx, sy);
                }
            }
        }
        const int nseg = kThreads / 32;
        double2 db = make_double2(0, 0);
        for (int q = gt; q < P; q += nthreads) {
            const double2 dq = d[q], v = cg_ld(b + q);
            db.x += dq.x * v.x - dq.y * v.y;
            db.y += dq.x * v.y + dq.y * v.x;
        }
        db = bsum(db, redz);
        if (tid == 0) w.zpart[blk] = db;
        if (!grid_barrier(w.sync, G)) return false;
        // phase A2: O b per sample
        for (int n = gt; n < N; n += nthreads) {
            double2 s = make_double2(0, 0);
            for (int j = 0; j < nseg; j++) {
                const double2 v = cg_ld(w.partA + (size_t)j * N + n);
                s = make_double2(s.x + v.x, s.y + v.y);
            }
            w.tmpN[n] = s;
        }
        db = sum_parts(w.zpart, G, redz);
        if (!grid_barrier(w.sync, G)) return false;
        // phase B: columns, 4 row groups x 64 columns per block
        const int c = tid % kColTile, rg = tid / kColTile, ngr = kThreads / kColTile;
        const int ntiles = (P + kColTile - 1) / kColTile;
        double2 pp = make_double2(0, 0);
        for (int tile = blk; tile < ntiles; tile += G) {
            const int q = tile * kColTile + c;
            double ax = 0, ay = 0;
            if (q < P) {
                // 8 rows in flight per thread: the pass is a stream over O
                int n = rg;
                for (; n + 7 * ngr < N; n += 8 * ngr) {
                    double2 o[8], v[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        o[u] = zld(O, (size_t)(n + u * ngr) * P + q);
                        v[u] = cg_ld(w.tmpN + n + u * ngr);
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        ax = fma(o[u].x, v[u].x, fma(o[u].y, v[u].y, ax));  // conj(o) v
                        ay = fma(o[u].x, v[u].y, fma(-o[u].y, v[u].x, ay));
                    }
                }
                for (; n < N; n += ngr) {
                    const double2 o = zld(O, (size_t)n * P + q), v = cg_ld(w.tmpN + n);
                    ax = fma(o.x, v.x, fma(o.y, v.y, ax));
                    ay = fma(o.x, v.y, fma(-o.y, v.x, ay));
                }
            }
            colred[tid] = make_double2(ax, ay);
            __syncthreads();
            if (rg == 0 && q < P) {
                double sx = 0, sy = 0;
                for (int g = 0; g < ngr; g++) {
                    sx += colred[g * kColTile + c].x;
                    sy += colred[g * kColTile + c].y;
                }
                const double2 dq = d[q], bq = cg_ld(b + q);
                const double f = diag[q] * (q < n_neural ? r1 : r1 + rd) + mxd * r2;
                // acc / norm - conj(d_q) (d . b), plus the shift
                double2 a;
                a.x = f * bq.x + sx / norm - (dq.x * db.x + dq.y * db.y);
                a.y = f * bq.y + sy / norm - (dq.x * db.y - dq.y * db.x);
                w.Ap[q] = a;
                if (want_pap) {
                    pp.x += bq.x * a.x + bq.y * a.y;
                    pp.y += bq.x * a.y - bq.y * a.x;
                }
            }
            __syncthreads();
        }
        if (want_pap) {
            pp = bsum(pp, redz);
            if (tid == 0) w.zpart[blk] = pp;
        }
        if (!grid_barrier(w.sync, G)) return false;
        if (want_pap) *pap = sum_parts(w.zpart, G, redz);
        return true;
    };

    if (w.minres) {
        // MINRES-QLP (Choi, Paige & Saunders; ACM TOMS 937), the solver of
        // optimizer.sr.method = minresqlp (zminresqlpModule.f90:42-1288 driven
        // by minresqlp_adapter.cpp:40-110): Lanczos on A with real
        // coefficients (A Hermitian), left reflections for the QR factors,
        // two right reflections per step for the LQ factors, MINRES updates
        // of x while the condition estimate stays below trancond and QLP
        // updates (minimum-length solution) after; x0 = 0.  The scalar
        // recurrence is carried redundantly by every thread (all blocks read
        // the same partial sums in the same order, so every copy agrees) and
        // the vectors are updated elementwise:
        //   v -> w.p, y -> w.Ap, r1 -> w.R1, r2 -> w.R2,
        //   w -> w.w2, wl -> w.w1, wl2 -> w.v, xl2 -> w.r.
        // Three grid barriers per iteration besides the operator's own.
        const double eps = 2.220446049250313e-16, maxxnorm = 1e7, trancond = 1e7, Acondlim = 1e15;
        double bl = 0;
        for (int q = gt; q < P; q += nthreads) {
            const double2 f = F[q];
            w.R1[q] = f;
            w.R2[q] = f;
            w.w1[q] = make_double2(0, 0);
            w.w2[q] = make_double2(0, 0);
            w.v[q] = make_double2(0, 0);
            w.r[q] = make_double2(0, 0);
            x[q] = make_double2(0, 0);
            bl += f.x * f.x + f.y * f.y;
        }
        bl = bsum(bl, redd);
        if (tid == 0) w.dpart[blk] = bl;
        bool mok = grid_barrier(w.sync, G);
        const double beta1 = mok ? sqrt(sum_parts(w.dpart, G, redd)) : 0.0;
        int istop = beta1 == 0 ? 3 : 0, itn = 0, qlp = 0;
        bool lastiter = false;
        double beta = 0, betal, betan = beta1, alfa, pnorm;
        double dbar, dlta, epln, eplnn = 0, dltan = 0, gbar = 0, dlta_qlp;
        double gama = 0, gamal = 0, gamal2 = 0, gamal3, gama_tmp;
        double tau = 0, taul = 0, taul2, phi = beta1, cs = -1, sn = 0, cr1 = -1, sr1 = 0, cr2 = -1, sr2 = 0;
        double vepln = 0, veplnl = 0, veplnl2 = 0, eta = 0, etal = 0, etal2 = 0;
        double u = 0, ul = 0, ul2 = 0, ul3 = 0, ul4;
        double xnorm = 0, xl2norm = 0, Anorm = 0, Acond = 1, Acondl = 1, gmin = 0, gminl = 0, gminl2;
        double rnorm = beta1, rnorml = beta1, relres = 1, relresl = 0, relAresl = 0, t1 = 2, t2 = 2;
        double gamal_qlp = 0, vepln_qlp = 0, gama_qlp = 0, ul_qlp = 0, u_qlp = 0;
        if (!mok) istop = -1;
        while (istop == 0) {
            itn++;
            // Lanczos step: v = y / beta, y = A v - (beta / betal) r1 - (alfa / beta) r2
            betal = beta;
            beta = betan;
            const double s = 1.0 / beta;
            for (int q = gt; q < P; q += nthreads) {
                const double2 r2 = cg_ld(w.R2 + q);
                w.p[q] = make_double2(s * r2.x, s * r2.y);
            }
            if (!(mok = grid_barrier(w.sync, G))) break;
            if (!(mok = aprod(w.p, false, nullptr))) break;
            double al = 0;
            const double cb = itn >= 2 ? beta / betal : 0.0;
            for (int q = gt; q < P; q += nthreads) {
                double2 y = cg_ld(w.Ap + q);
                const double2 r1 = cg_ld(w.R1 + q), v = cg_ld(w.p + q);
                y.x -= cb * r1.x;
                y.y -= cb * r1.y;
                w.Ap[q] = y;
                al += v.x * y.x + v.y * y.y;
            }
            al = bsum(al, redd);
            if (tid == 0) w.dpart[blk] = al;
            if (!(mok = grid_barrier(w.sync, G))) break;
            alfa = sum_parts(w.dpart, G, redd);
            double bb = 0;
            const double ca = alfa / beta;
            for (int q = gt; q < P; q += nthreads) {
                double2 y = cg_ld(w.Ap + q);
                const double2 r2 = cg_ld(w.R2 + q);
                y.x -= ca * r2.x;
                y.y -= ca * r2.y;
                w.R1[q] = r2;
                w.R2[q] = y;
                bb += y.x * y.x + y.y * y.y;
            }
            bb = bsum(bb, redd);
            if (tid == 0) w.zpart[blk] = make_double2(bb, 0);
            if (!(mok = grid_barrier(w.sync, G))) break;
            betan = sqrt(sum_parts(w.zpart, G, redz).x);
            pnorm = itn == 1 ? hypot(alfa, betan) : norm3d(beta, alfa, betan);
            // previous left reflection
            dbar = dltan;
            dlta = cs * dbar + sn * alfa;
            epln = eplnn;
            gbar = sn * dbar - cs * alfa;
            eplnn = sn * betan;
            dltan = -cs * betan;
            dlta_qlp = dlta;
            // current left reflection
            gamal3 = gamal2;
            gamal2 = gamal;
            gamal = gama;
            symortho(gbar, betan, cs, sn, gama);
            gama_tmp = gama;
            taul2 = taul;
            taul = tau;
            tau = cs * phi;
            phi = sn * phi;
            // previous right reflection P_{k-2,k}
            if (itn > 2) {
                veplnl2 = veplnl;
                etal2 = etal;
                etal = eta;
                const double dt = sr2 * vepln - cr2 * dlta;
                veplnl = cr2 * vepln + sr2 * dlta;
                dlta = dt;
                eta = sr2 * gama;
                gama = -cr2 * gama;
            }
            // current right reflection P_{k-1,k}
            if (itn > 1) {
                double g;
                symortho(gamal, dlta, cr1, sr1, g);
                gamal = g;
                vepln = sr1 * gama;
                gama = -cr1 * gama;
            }
            // solution norm
            ul4 = ul3;
            ul3 = ul2;
            if (itn > 2) ul2 = (taul2 - etal2 * ul4 - veplnl2 * ul3) / gamal2;
            if (itn > 1) ul = (taul - etal * ul3 - veplnl * ul2) / gamal;
            const double xt = norm3d(xl2norm, ul2, ul);
            if (fabs(gama) > 0 && xt < maxxnorm) {
                u = (tau - eta * ul2 - vepln * ul) / gama;
                if (relAresl < relresl && hypot(xt, u) > maxxnorm) {
                    u = 0;
                    istop = 12;
                }
            } else {
                u = 0;
                istop = 14;
            }
            xl2norm = hypot(xl2norm, ul2);
            xnorm = norm3d(xl2norm, ul, u);
            if (Acond < trancond && istop == 0 && qlp == 0) {
                // MINRES updates
                const bool upd = xnorm < maxxnorm;
                const double ig = fabs(gama_tmp) > 0 ? 1.0 / gama_tmp : 0.0;
                for (int q = gt; q < P; q += nthreads) {
                    const double2 v = cg_ld(w.p + q), a1 = cg_ld(w.w1 + q), a2 = cg_ld(w.w2 + q);
                    double2 wn = a2;
                    if (ig != 0)
                        wn = make_double2((v.x - epln * a1.x - dlta_qlp * a2.x) * ig,
                                          (v.y - epln * a1.y - dlta_qlp * a2.y) * ig);
                    w.v[q] = a1;
                    w.w1[q] = a2;
                    w.w2[q] = wn;
                    if (upd) {
                        double2 xq = cg_ld(x + q);
                        xq.x += tau * wn.x;
                        xq.y += tau * wn.y;
                        x[q] = xq;
                    }
                }
                if (!upd) {
                    istop = 12;
                    lastiter = true;
                }
            } else {
                // MINRES-QLP updates
                qlp++;
                const bool first = qlp == 1;
                for (int q = gt; q < P; q += nthreads) {
                    double2 W = cg_ld(w.w2 + q), WL = cg_ld(w.w1 + q), WL2 = cg_ld(w.v + q);
                    double2 XL2 = cg_ld(w.r + q);
                    const double2 v = cg_ld(w.p + q), xq = cg_ld(x + q);
                    if (first) {
                        // transfer from the MINRES vectors
                        XL2 = make_double2(0, 0);
                        if (itn > 1) {
                            if (itn > 3)
                                WL2 = make_double2(gamal3 * WL2.x + veplnl2 * WL.x + etal * W.x,
                                                   gamal3 * WL2.y + veplnl2 * WL.y + etal * W.y);
                            if (itn > 2)
                                WL = make_double2(gamal_qlp * WL.x + vepln_qlp * W.x,
                                                  gamal_qlp * WL.y + vepln_qlp * W.y);
                            W = make_double2(gama_qlp * W.x, gama_qlp * W.y);
                            XL2 = make_double2(xq.x - ul_qlp * WL.x - u_qlp * W.x, xq.y - ul_qlp * WL.y - u_qlp * W.y);
                        }
                    }
                    if (itn == 1) {
                        WL2 = WL;
                        WL = make_double2(sr1 * v.x, sr1 * v.y);
                        W = make_double2(-cr1 * v.x, -cr1 * v.y);
                    } else if (itn == 2) {
                        WL2 = WL;
                        WL = make_double2(cr1 * W.x + sr1 * v.x, cr1 * W.y + sr1 * v.y);
                        W = make_double2(sr1 * W.x - cr1 * v.x, sr1 * W.y - cr1 * v.y);
                    } else {
                        const double2 a = WL, b = W;
                        const double2 wt = make_double2(sr2 * a.x - cr2 * v.x, sr2 * a.y - cr2 * v.y);
                        WL2 = make_double2(cr2 * a.x + sr2 * v.x, cr2 * a.y + sr2 * v.y);
                        WL = make_double2(cr1 * b.x + sr1 * wt.x, cr1 * b.y + sr1 * wt.y);
                        W = make_double2(sr1 * b.x - cr1 * wt.x, sr1 * b.y - cr1 * wt.y);
                    }
                    XL2 = make_double2(XL2.x + ul2 * WL2.x, XL2.y + ul2 * WL2.y);
                    w.w2[q] = W;
                    w.w1[q] = WL;
                    w.v[q] = WL2;
                    w.r[q] = XL2;
                    x[q] = make_double2(XL2.x + ul * WL.x + u * W.x, XL2.y + ul * WL.y + u * W.y);
                }
            }
            // next right reflection P_{k-1,k+1}
            gamal_qlp = gamal;
            symortho(gamal_qlp, eplnn, cr2, sr2, gamal);
            vepln_qlp = vepln;
            gama_qlp = gama;
            ul_qlp = ul;
            u_qlp = u;
            // norm and condition estimates
            const double ag = fabs(gama);
            Anorm = fmax(fmax(Anorm, pnorm), fmax(fabs(gamal), ag));
            if (itn == 1) {
                gmin = ag;
                gminl = gmin;
            } else {
                gminl2 = gminl;
                gminl = gmin;
                gmin = fmin(gminl2, fmin(fabs(gamal), ag));
            }
            Acondl = Acond;
            Acond = Anorm / gmin;
            rnorml = rnorm;
            relresl = relres;
            if (istop != 14) rnorm = fabs(phi);
            relres = rnorm / (Anorm * xnorm + beta1);
            relAresl = hypot(gbar, dltan) / Anorm;
            // stopping rules in the published order
            const double epsx = Anorm * xnorm * eps;
            if (istop == 0 || istop == 14) {
                t1 = 1 + relres;
                t2 = 1 + relAresl;
            }
            if (t1 <= 1) istop = 5;
            else if (t2 <= 1) istop = 7;
            else if (relres <= rtol) istop = 4;
            else if (relAresl <= rtol) istop = 6;
            else if (epsx >= beta1) istop = 2;
            else if (xnorm >= maxxnorm) istop = 12;
            else if (Acond >= Acondlim || Acond >= 0.1 / eps) istop = 13;
            else if (itn >= max_it) istop = 8;
            else if (betan < eps) istop = 1;
            // the last step's estimates are not kept for these stops
            if (istop == 6 || istop == 7 || istop == 12 || istop == 13) lastiter = true;
            if (istop != 0 && lastiter) {
                itn--;
                Acond = Acondl;
                rnorm = rnorml;
                relres = relresl;
            }
        }
        if (blk == 0 && tid == 0) {
            res->iterations = itn;
            res->residual = rnorm;
            res->istop = istop;
            res->acond = Acond;
            res->qlp_iterations = qlp;
            if (!mok) res->status = -2;
        }
        return;
    }

    bool ok = aprod(x, false, nullptr);
    // r = F - A x0, p = r
    double rl = 0;
    if (ok) {
        for (int q = gt; q < P; q += nthreads) {
            const double2 aq = cg_ld(w.Ap + q);
            const double2 rq = make_double2(F[q].x - aq.x, F[q].y - aq.y);
            w.r[q] = rq;
            w.p[q] = rq;
            rl += rq.x * rq.x + rq.y * rq.y;
        }
        rl = bsum(rl, redd);
        if (tid == 0) w.dpart[blk] = rl;
        ok = grid_barrier(w.sync, G);
    }
    double rsold = ok ? sum_parts(w.dpart, G, redd) : 0.0, rs = rsold;
    int itn = 0;
    if (ok) {
        for (itn = 0; itn < max_it; itn++) {
            double2 pap;
            if (!(ok = aprod(w.p, true, &pap))) break;
            // alpha = rsold / (p^H A p)
            const double den = pap.x * pap.x + pap.y * pap.y;
            const double ax = rsold * pap.x / den, ay = -rsold * pap.y / den;
            rl = 0;
            for (int q = gt; q < P; q += nthreads) {
                const double2 pq = cg_ld(w.p + q), aq = cg_ld(w.Ap + q);
                double2 xq = cg_ld(x + q), rq = cg_ld(w.r + q);
                xq.x += ax * pq.x - ay * pq.y;
                xq.y += ax * pq.y + ay * pq.x;
                rq.x -= ax * aq.x - ay * aq.y;
                rq.y -= ax * aq.y + ay * aq.x;
                x[q] = xq;
                w.r[q] = rq;
                rl += rq.x * rq.x + rq.y * rq.y;
            }
            rl = bsum(rl, redd);
            if (tid == 0) w.dpart[blk] = rl;
            if (!(ok = grid_barrier(w.sync, G))) break;
            rs = sum_parts(w.dpart, G, redd);
            if (rs < rtol) break;
            const double beta = rs / rsold;
            for (int q = gt; q < P; q += nthreads) {
                const double2 rq = cg_ld(w.r + q), pq = cg_ld(w.p + q);
                w.p[q] = make_double2(rq.x + beta * pq.x, rq.y + beta * pq.y);
            }
            rsold = rs;
            if (!(ok = grid_barrier(w.sync, G))) break;
        }
    }
    if (blk == 0 && tid == 0) {
        res->iterations = itn;
        res->residual = rs;
        if (!ok) res->status = -2;
    }
}

// diag_p = (1/(N-1)) sum_n |O_np - d_p|^2 (the unbiased var(O) of the
// aggregator, aggregator.cpp:84-164) and per-block maxima.
template <typename TO>
__global__ void __launch_bounds__(kThreads) var_diag_kernel(const TO* __restrict__ O, const double2* __restrict__ d,
                                                            int N, int P, double* diag, double* maxpart,
                                                            const double* vfac) {
    __shared__ double colred[kThreads];
    __shared__ double red[kThreads / 32];
    const int tid = threadIdx.x, c = tid % kColTile, rg = tid / kColTile, ngr = kThreads / kColTile;
    const int ntiles = (P + kColTile - 1) / kColTile;
    double mx = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int q = tile * kColTile + c;
        double s = 0;
        if (q < P) {
            const double2 dq = d[q];
            for (int n = rg; n < N; n += ngr) {
                const double2 o = zld(O, (size_t)n * P + q);
                const double ex = o.x - dq.x, ey = o.y - dq.y;
                s = fma(ex, ex, fma(ey, ey, s));
            }
        }
        colred[tid] = s;
        __syncthreads();
        if (rg == 0 && q < P) {
            double t = 0;
            for (int g = 0; g < ngr; g++) t += colred[g * kColTile + c];
            if (vfac)
                t = t / (double)N * *vfac;
            else
                t /= (double)N - 1.0;
            diag[q] = t;
            mx = fmax(mx, t);
        }
        __syncthreads();
    }
    const int lane = tid & 31, w = tid >> 5;
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[w] = mx;
    __syncthreads();
    if (tid == 0) {
        double m = red[0];
        for (int i = 1; i < kThreads / 32; i++) m = fmax(m, red[i]);
        maxpart[blockIdx.x] = m;
    }
}

__global__ void max_parts_kernel(const double* maxpart, int n, double* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double m = maxpart[0];
        for (int i = 1; i < n; i++) m = fmax(m, maxpart[i]);
        *out = m;
    }
}

template <typename TO> const void* cg_fn() { return reinterpret_cast<const void*>(cg_mfree_kernel<TO>); }

// CG (cg1 semantics, cg_solver.cpp:260-334) on a formed regularised S with
// one grid barrier per iteration.  Every block keeps full copies of p, r and
// x in shared memory and updates them itself, with the same sums in the same
// order as every other block, so alpha and beta agree bit for bit across the
// grid; the only data exchanged through global memory is A p, one row per
// warp, written to one of two buffers by iteration parity (a block one
// iteration ahead writes the other buffer while slower blocks still read).
__global__ void __launch_bounds__(kThreads) cg_dense1_kernel(const double2* __restrict__ S,
                                                             const double2* __restrict__ F, double2* x, int P,
                                                             int max_it, double rtol, MfreeWork w, CgResultDev* res,
                                                             int cache_rows) {
    extern __shared__ double2 sv[];
    double2 *p = sv, *r = sv + P, *xs = sv + 2 * P;
    // cache_rows: every warp owns at most one row of S (the grid has at
    // least P warps) and keeps it in shared memory for the whole solve
    double2* srow = sv + 3 * P + (size_t)(threadIdx.x >> 5) * P;
    __shared__ double redd[kThreads / 32];
    __shared__ double2 redz[kThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, G = gridDim.x, blk = blockIdx.x;
    const int gw = blk * (kThreads / 32) + (tid >> 5), nwarps = G * (kThreads / 32);
    if (blk == 0 && tid == 0) {
        res->status = 0;
        res->istop = 0;
        res->qlp_iterations = 0;
        res->acond = 0;
    }
    if (cache_rows && gw < P)
        for (int q = lane; q < P; q += 32) srow[q] = __ldg(S + (size_t)gw * P + q);
    // rows of S times a shared-memory vector into a global buffer
    auto matvec = [&](const double2* v, double2* out) {
        for (int row = gw; row < P; row += nwarps) {
            const double2* Sr = cache_rows ? srow : S + (size_t)row * P;
            double ax = 0, ay = 0;
            int q = lane;
            for (; q + 96 < P; q += 128) {
                double2 a[4], b[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    a[u] = cache_rows ? Sr[q + 32 * u] : __ldg(Sr + q + 32 * u);
                    b[u] = v[q + 32 * u];
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    ax = fma(a[u].x, b[u].x, fma(-a[u].y, b[u].y, ax));
                    ay = fma(a[u].x, b[u].y, fma(a[u].y, b[u].x, ay));
                }
            }
            for (; q < P; q += 32) {
                const double2 a = cache_rows ? Sr[q] : __ldg(Sr + q), b = v[q];
                ax = fma(a.x, b.x, fma(-a.y, b.y, ax));
                ay = fma(a.x, b.y, fma(a.y, b.x, ay));
            }
            ax = warp_sum(ax);
            ay = warp_sum(ay);
            if (lane == 0) out[row] = make_double2(ax, ay);
        }
    };
    for (int q = tid; q < P; q += kThreads) xs[q] = x[q];
    __syncthreads();
    matvec(xs, w.Ap);
    bool ok = grid_barrier(w.sync, G);
    double rs = 0.0;
    int itn = 0;
    if (ok) {
        // r = F - A x0, p = r
        double rl = 0;
        for (int q = tid; q < P; q += kThreads) {
            const double2 aq = cg_ld(w.Ap + q);
            const double2 rq = make_double2(F[q].x - aq.x, F[q].y - aq.y);
            r[q] = rq;
            p[q] = rq;
            rl += rq.x * rq.x + rq.y * rq.y;
        }
        double rsold = bsum(rl, redd);
        rs = rsold;
        for (itn = 0; itn < max_it; itn++) {
            double2* ab = (itn & 1) ? w.Ap : w.R1;  // A x0 went to w.Ap
            matvec(p, ab);
            if (!(ok = grid_barrier(w.sync, G))) break;
            // alpha = rsold / (p^H A p)
            double2 pp = make_double2(0, 0);
            for (int q = tid; q < P; q += kThreads) {
                const double2 aq = cg_ld(ab + q), pq = p[q];
                pp.x += pq.x * aq.x + pq.y * aq.y;
                pp.y += pq.x * aq.y - pq.y * aq.x;
            }
            const double2 pap = bsum(pp, redz);
            const double den = pap.x * pap.x + pap.y * pap.y;
            const double ax = rsold * pap.x / den, ay = -rsold * pap.y / den;
            double rl2 = 0;
            for (int q = tid; q < P; q += kThreads) {
                const double2 pq = p[q], aq = cg_ld(ab + q);
                double2 xq = xs[q], rq = r[q];
                xq.x += ax * pq.x - ay * pq.y;
                xq.y += ax * pq.y + ay * pq.x;
                rq.x -= ax * aq.x - ay * aq.y;
                rq.y -= ax * aq.y + ay * aq.x;
                xs[q] = xq;
                r[q] = rq;
                rl2 += rq.x * rq.x + rq.y * rq.y;
            }
            rs = bsum(rl2, redd);
            if (rs < rtol) break;
            const double beta = rs / rsold;
            for (int q = tid; q < P; q += kThreads) {
                const double2 rq = r[q], pq = p[q];
                p[q] = make_double2(rq.x + beta * pq.x, rq.y + beta * pq.y);
            }
            rsold = rs;
            __syncthreads();
        }
    }
    __syncthreads();
    if (blk == 0) {
        for (int q = tid; q < P; q += kThreads) x[q] = xs[q];
        if (tid == 0) {
            res->iterations = itn;
            res->residual = rs;
            if (!ok) res->status = -2;
        }
    }
}

}  // namespace

__global__ void init_sync_kernel(MfreeSync* sync, uint32_t extra, uint32_t cap) {
    sync->count = 0;
    sync->gen = 0;
    sync->bad = 0;
    sync->extra = extra;
    sync->spin_cap = cap;
}

cudaError_t launch_init_sync(MfreeSync* sync, cudaStream_t st) {
    const bool stall = test_fault() == 1;
    init_sync_kernel<<<1, 1, 0, st>>>(sync, stall ? 1u : 0u, stall ? 1024u : 0u);
    return cudaGetLastError();
}

cudaError_t mfree_plan(int N, int P, MfreePlan* pl) {
    int dev = 0, sms = 148, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return cudaErrorNotSupported;
    // the smaller of the two instantiations' residency bounds
    int b32 = 0, b64 = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b32, cg_mfree_kernel<float2>, kThreads, 0);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b64, cg_mfree_kernel<double2>, kThreads, 0);
    if (e != cudaSuccess) return e;
    per_sm = b32 < b64 ? b32 : b64;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    if (per_sm > 2) per_sm = 2;
    pl->blocks = sms * per_sm;
    // formed S (N == 1): one warp per row of S is all the mat-vec can use,
    // and fewer blocks make every grid barrier cheaper
    if (N == 1) {
        const int want = (P + kThreads / 32 - 1) / (kThreads / 32);
        if (want < pl->blocks) pl->blocks = want < 1 ? 1 : want;
    }
    pl->nseg = kThreads / 32;  // column slices of the O b pass (one per warp of a block)
    pl->lseg = (P + pl->nseg - 1) / pl->nseg;
    pl->diag_blocks = pl->blocks;
    return cudaSuccess;
}

size_t mfree_work_bytes(int N, int P, const MfreePlan& pl) {
    return ((size_t)8 * P + N + (size_t)pl.nseg * N + 2 * (size_t)pl.blocks) * sizeof(double2) +
           (size_t)pl.blocks * sizeof(double) * 2 + sizeof(MfreeSync) + 256;
}

MfreeWork mfree_carve(void* base, int N, int P, const MfreePlan& pl) {
    MfreeWork w{};
    auto* z = reinterpret_cast<double2*>(base);
    w.r = z;
    w.p = w.r + P;
    w.Ap = w.p + P;
    w.R1 = w.Ap + P;
    w.R2 = w.R1 + P;
    w.w1 = w.R2 + P;
    w.w2 = w.w1 + P;
    w.v = w.w2 + P;
    w.tmpN = w.v + P;
    w.partA = w.tmpN + N;
    w.zpart = w.partA + (size_t)pl.nseg * N;
    auto* dd = reinterpret_cast<double*>(w.zpart + 2 * (size_t)pl.blocks);
    w.dpart = dd;
    w.maxpart = dd + pl.blocks;
    w.sync = reinterpret_cast<MfreeSync*>(reinterpret_cast<uintptr_t>(w.maxpart + pl.blocks) + 255 & ~uintptr_t(255));
    w.nseg = pl.nseg;
    w.lseg = pl.lseg;
    return w;
}

cudaError_t launch_max_diag(const double* diag, int P, double* max_diag, cudaStream_t st) {
    max_parts_kernel<<<1, 32, 0, st>>>(diag, P, max_diag);
    return cudaGetLastError();
}

cudaError_t launch_cg_dense_coop(const double2* A, const double2* b, double2* x, int P, int max_it, double rtol,
                                 const MfreePlan& pl, const MfreeWork& w, CgResultDev* res, cudaStream_t st) {
    cudaError_t e = launch_init_sync(w.sync, st);
    if (e != cudaSuccess) return e;
    if (!w.minres) {
        // CG: the one-barrier kernel, p, r and x of every block in shared
        // memory, and each warp's row of S too when the rows fit
        const int base_smem = 3 * P * (int)sizeof(double2);
        const int row_smem = (kThreads / 32) * P * (int)sizeof(double2);
        const void* fn = reinterpret_cast<const void*>(cg_dense1_kernel);
        int dev = 0, sms = 148, per_sm = 0, smem_max = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        const int rows_blocks = (P + kThreads / 32 - 1) / (kThreads / 32);  // one row per warp
        int cache = base_smem + row_smem <= smem_max - 8 * 1024 ? 1 : 0;
        int smem = base_smem + (cache ? row_smem : 0);
        if ((e = ensure_dynamic_smem(fn, smem)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_dense1_kernel, kThreads, smem)) !=
            cudaSuccess)
            return e;
        if (cache && rows_blocks > sms * per_sm) {  // not every row gets its own warp
            cache = 0;
            smem = base_smem;
            if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_dense1_kernel, kThreads, smem)) !=
                cudaSuccess)
                return e;
        }
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        int blocks = std::min(sms * per_sm, rows_blocks);
        blocks = std::max(1, blocks);
        MfreeWork wk = w;
        const double2* S = A;
        const double2* F = b;
        double2* xo = x;
        CgResultDev* r = res;
        void* args[] = {&S, &F, &xo, &P, &max_it, &rtol, &wk, &r, &cache};
        return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kThreads), args, smem, st);
    }
    MfreeWork wk = w;
    wk.S = A;
    const double2* O = nullptr;
    const double2* d = nullptr;
    const double* diag = nullptr;
    const double* mx = nullptr;
    const ScheduleDev* sch = nullptr;
    double norm = 1.0, z = 0.0;
    int N = 1, n_neural = P;
    CgResultDev* r = res;
    const void* args[] = {&O, &d, &norm, &N, &P, &n_neural, &b, &x, &diag, &mx, &sch, &z, &z, &z,
                          &max_it, &rtol, &wk, &r};
    return cudaLaunchCooperativeKernel(cg_fn<double2>(), dim3(pl.blocks), dim3(kThreads), const_cast<void**>(args), 0,
                                       st);
}

cudaError_t launch_var_diag(const void* O, int fp64, const double2* d, int N, int P, const MfreePlan& pl,
                            const MfreeWork& w, double* diag, double* max_diag, cudaStream_t st,
                            const double* vfac) {
    if (fp64)
        var_diag_kernel<double2>
            <<<pl.diag_blocks, kThreads, 0, st>>>((const double2*)O, d, N, P, diag, w.maxpart, vfac);
    else
        var_diag_kernel<float2><<<pl.diag_blocks, kThreads, 0, st>>>((const float2*)O, d, N, P, diag, w.maxpart, vfac);
    max_parts_kernel<<<1, 32, 0, st>>>(w.maxpart, pl.diag_blocks, max_diag);
    return cudaGetLastError();
}

cudaError_t launch_cg_mfree(const void* O, int fp64, const double2* d, double norm, int N, int P, int n_neural,
                            const double2* F, double2* x, const double* diag, const double* max_diag,
                            const ScheduleDev* sch, double r1, double r2, double rd, int max_it, double rtol,
                            const MfreePlan& pl, const MfreeWork& w, CgResultDev* res, cudaStream_t st) {
    // barrier state: count 0, no failure
    cudaError_t e = launch_init_sync(w.sync, st);
    if (e != cudaSuccess) return e;
    MfreeWork wk = w;
    CgResultDev* r = res;
    const void* args[] = {&O, &d, &norm, &N, &P, &n_neural, &F, &x, &diag, &max_diag, &sch, &r1, &r2, &rd,
                          &max_it, &rtol, &wk, &r};
    return cudaLaunchCooperativeKernel(fp64 ? cg_fn<double2>() : cg_fn<float2>(), dim3(pl.blocks), dim3(kThreads),
                                       const_cast<void**>(args), 0, st);
}

}  // namespace rbmnqs
