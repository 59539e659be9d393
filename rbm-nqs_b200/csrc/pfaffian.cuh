// pfaffian.cuh -- the Pfaffian pair-wavefunction factor (machine/pfaffian.cpp)
// on the GPU: one warp per configuration, up to 32 sites.  FP64 throughout.
//
//   X_ij    = sgn(bs_ij) fs[|bs_ij| - 1, 2 s_i + s_j]    (pfaffian.cpp:127-137)
//   context = X^{-1}, antisymmetrised                    (pfaffian.cpp:284-297)
//   ratio   = (-1)^{m(m+1)/2} Pf(C^{-1}) for m flips,
//             C^{-1} = C0 + tmp - tmp^T, tmp = B^T X^{-1} B / 2
//   update  X^{-1} += X^{-1}B C B^T X^{-1} (antisymmetric)  (pfaffian.cpp:314-397)
//   d/dfs   d[|bs_ij| - 1, 2 s_i + s_j] -/+= X^{-1}_ij, j < i (pfaffian.cpp:399-415)
//
// X^{-1} lives in a per-warp shared-memory matrix (leading dimension 33,
// conflict-free for both row and column walks).  The fresh inverse is a
// Gauss-Jordan elimination with partial (row) pivoting in which rows stay in
// place and the pivot row of column k is recorded; the inverse then comes
// out with rows and columns permuted, S[p_k][j] = X^{-1}[k][p_j], and is
// unscrambled through a second per-warp n x n buffer in the same pass that
// antisymmetrises it.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace rbmnqs {

constexpr int kPfMaxSites = 32;
constexpr int kPfMaxFlips = 4;

struct PfDev {
    int n = 0;        // sites (<= 32); 0 = no Pfaffian factor
    int n_indep = 0;  // independent pair classes
    int refresh = 0;  // fresh context every `refresh` accepted moves (0: never)
    const int16_t* bs = nullptr;       // [n][n] row-major bs_(i, j), signed 1-based class
    const double2* fs = nullptr;       // [4][n_indep]: fs[c * n_indep + a] = fs_(a, c)
    const int* pair_ptr = nullptr;     // [n_indep + 1] CSR over classes
    const uint32_t* pairs = nullptr;   // (i << 16) | (j << 8) | (bs_ij > 0), i > j
    double2* scratch = nullptr;        // sampler: [warps][32 * 32] unscramble buffers (global)
};

// Per-warp staging in shared memory.
struct PfStage {
    double2 B[kPfMaxSites][kPfMaxFlips];       // dense columns of B
    double2 IB[kPfMaxSites][2 * kPfMaxFlips];  // rows of X^{-1} B
    double2 C[2 * kPfMaxFlips][2 * kPfMaxFlips];
    int piv[kPfMaxSites];                      // Gauss-Jordan pivot row of each column
};

// smem leading dimension of an n x n FP64 complex matrix: 33 keeps a column
// walk (lane i, fixed j) free of bank conflicts
constexpr int kPfLd = 33;
constexpr int kPfMatBytes = kPfMaxSites * kPfLd * 16;

__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// acc + a * b
__device__ __forceinline__ double2 zfma(double2 a, double2 b, double2 acc) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}
__device__ __forceinline__ double2 zscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double zabs2(double2 a) { return fma(a.x, a.x, a.y * a.y); }
// 1 / z (0 for z == 0, which only a singular pair matrix produces)
__device__ __forceinline__ double2 zrcp(double2 z) {
    const double d = zabs2(z);
    if (d == 0.0) return make_double2(0.0, 0.0);
    const double r = 1.0 / d;
    return make_double2(z.x * r, -z.y * r);
}
__device__ __forceinline__ double2 zdiv(double2 a, double2 b) { return zmul(a, zrcp(b)); }
__device__ __forceinline__ double2 zshfl(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// pfaffian::a (pfaffian.cpp:127-137): element (i, j) of X with bits fi, fj
// toggled on sites i, j.  bits: site q down iff bit q set.
__device__ __forceinline__ double2 pf_elem(const PfDev& p, uint32_t bits, int i, int j, int fi, int fj) {
    if (i == j) return make_double2(0.0, 0.0);
    const int b = p.bs[i * p.n + j];
    const int bi = ((bits >> i) & 1) ^ fi, bj = ((bits >> j) & 1) ^ fj;
    const int sp = j < i ? (bi << 1) + bj : (bj << 1) + bi;
    const double2 v = __ldg(&p.fs[sp * p.n_indep + (b < 0 ? -b : b) - 1]);
    return b < 0 ? make_double2(-v.x, -v.y) : v;
}

// Warp argmax of v (ties: lowest lane).
__device__ __forceinline__ int warp_argmax(double v) {
    int who = threadIdx.x & 31;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int ow = __shfl_xor_sync(0xffffffffu, who, off);
        if (ov > v || (ov == v && ow < who)) {
            v = ov;
            who = ow;
        }
    }
    return who;
}

// Gauss-Jordan inverse of X (configuration `bits`) in the n x n workspace A
// (leading dimension LD; shared or global memory), partial (row) pivoting
// with rows kept in place: afterwards row piv[k] of A holds X^{-1}[k][piv[j]]
// in column j.  Lane = column for the row operations, lane = row for the
// pivot search.  The full 32 x 32 block is written (rows / columns >= n
// zero).  Two elimination steps share one pass over the rows: the second
// pivot column is updated by the first step in registers, and each row takes
// both rank-1 updates between one load and one store -- the operations and
// their order are those of two single steps, so the result is the same to
// the bit, with half the row traffic (the workspace of the sweep is global
// memory, whose stores go through to L2).  The two pivot columns reach the
// row loop through fb (2 x 32 entries of per-warp shared memory, read as
// broadcasts), the column-(k + 1) special case through the multiplier of the
// first update.  LD is a compile-time constant so that the row updates can
// be issued back to back.  The loops stay rolled: the elimination runs
// between proposals of the other warps of the SM, whose loop must stay in
// the instruction cache.  Warp-collective.
template <int LD>
__device__ __forceinline__ void pf_gauss_jordan(const PfDev& p, uint32_t bits, int lane, double2* A, int* piv,
                                                double2* fb) {
    constexpr int ld = LD;
    const int n = p.n;
    const double2 zero = make_double2(0.0, 0.0);
#pragma unroll 2
    for (int i = 0; i < kPfMaxSites; i++)
        A[i * ld + lane] = (i < n && lane < n) ? pf_elem(p, bits, i, lane, 0, 0) : zero;
    __syncwarp();
    uint32_t used = 0;
    int k = 0;
#pragma unroll 1
    for (; k + 1 < n; k += 2) {
        // step k: pivot row p1 of column k (c0), normalised row rp1
        const double2 c0 = lane < n ? A[lane * ld + k] : zero;
        const double2 c1 = lane < n ? A[lane * ld + k + 1] : zero;
        const int p1 = warp_argmax((lane < n && !((used >> lane) & 1u)) ? zabs2(c0) : -1.0);
        used |= 1u << p1;
        if (lane == 0) piv[k] = p1;
        const double2 ip1 = zrcp(zshfl(c0, p1));
        double2 rp1 = zero;
        if (lane < n) rp1 = lane == k ? ip1 : zmul(A[p1 * ld + lane], ip1);
        // column k + 1 after step k (row p1 holds rp1)
        const double2 r1k1 = zshfl(rp1, k + 1);
        const double2 c1u = lane == p1 ? r1k1 : zsub(c1, zmul(c0, r1k1));
        fb[lane] = c0;
        fb[kPfMaxSites + lane] = c1u;
        // step k + 1: pivot row p2 of the updated column, normalised row rp2
        const int p2 = warp_argmax((lane < n && !((used >> lane) & 1u)) ? zabs2(c1u) : -1.0);
        used |= 1u << p2;
        if (lane == 0) piv[k + 1] = p2;
        const double2 ip2 = zrcp(zshfl(c1u, p2));
        const double2 f1p2 = zshfl(c0, p2), f2p1 = zshfl(c1u, p1);
        double2 rp2 = zero, r1p = zero;
        if (lane < n) {
            const double2 a1 = zsub(lane == k ? zero : A[p2 * ld + lane], zmul(f1p2, rp1));
            rp2 = lane == k + 1 ? ip2 : zmul(a1, ip2);
            r1p = zsub(lane == k + 1 ? zero : rp1, zmul(f2p1, rp2));
        }
        __syncwarp();
        // the other rows: a - f1 rp1 - f2 rp2, with a = 0 in columns k and
        // k + 1 and, in column k + 1, the first update's result discarded
        // (rp1 there taken as 0: 0 - f1 0 = +0, as the discarded value)
        const bool keep = lane != k && lane != k + 1;
        const double2 rp1e = lane == k + 1 ? zero : rp1;
        if (lane < n) {
#pragma unroll 2
            for (int i = 0; i < n; i++) {
                if (i == p1 || i == p2) continue;  // uniform
                const double2 f1 = fb[i], f2 = fb[kPfMaxSites + i];
                const double2 a = keep ? A[i * ld + lane] : zero;
                A[i * ld + lane] = zsub(zsub(a, zmul(f1, rp1e)), zmul(f2, rp2));
            }
            A[p2 * ld + lane] = rp2;
            A[p1 * ld + lane] = r1p;
        }
        __syncwarp();
    }
    if (k < n) {  // odd n: one single step
        const double2 fcol = lane < n ? A[lane * ld + k] : zero;
        const int pr = warp_argmax((lane < n && !((used >> lane) & 1u)) ? zabs2(fcol) : -1.0);
        used |= 1u << pr;
        if (lane == 0) piv[k] = pr;
        const double2 ip = zrcp(zshfl(fcol, pr));
        double2 rp = zero;
        if (lane < n) {
            rp = lane == k ? ip : zmul(A[pr * ld + lane], ip);
            A[pr * ld + lane] = rp;
        }
        for (int i = 0; i < n; i++) {
            if (i == pr) continue;
            const double2 f = zshfl(fcol, i);
            if (lane < n) A[i * ld + lane] = zsub(lane == k ? zero : A[i * ld + lane], zmul(f, rp));
        }
        __syncwarp();
    }
}

// Fresh context (pfaffian::get_context): A <- the antisymmetrised X^{-1} of
// configuration `bits`.  A: the warp's n x n shared-memory matrix (leading
// dimension kPfLd); scr: a second per-warp n x n buffer (global or shared,
// leading dimension sld) for the unscramble.  Warp-collective.
__device__ __forceinline__ void pf_fresh(const PfDev& p, uint32_t bits, int lane, double2* A, PfStage& st,
                                         double2* scr, int sld) {
    const int n = p.n;
    pf_gauss_jordan<kPfLd>(p, bits, lane, A, st.piv, &st.IB[0][0]);
    // unscramble: row p_k of A holds X^{-1}[k][p_j] in column j
    if (lane < n) {
        const int pj = st.piv[lane];
        for (int k = 0; k < n; k++) scr[k * sld + pj] = A[st.piv[k] * kPfLd + lane];
    }
    __syncwarp();
    // antisymmetrise (pfaffian.cpp:290-293)
    if (lane < n)
        for (int i = 0; i < n; i++) {
            const double2 a = scr[i * sld + lane], b = scr[lane * sld + i];
            A[i * kPfLd + lane] = make_double2(0.5 * (a.x - b.x), 0.5 * (a.y - b.y));
        }
    __syncwarp();
}

// Pfaffian of the antisymmetric m2 x m2 matrix st.C (upper triangle used),
// m2 = 2 or 4 in closed form; 6 and 8 by Parlett-Reid elimination on lane 0
// (the matrix is overwritten).  Result valid on every lane.
__device__ __forceinline__ double2 pf_small(PfStage& st, int m2, int lane) {
    const auto& C = st.C;
    if (m2 == 2) return C[0][1];
    if (m2 == 4)
        return zadd(zsub(zmul(C[0][1], C[2][3]), zmul(C[0][2], C[1][3])), zmul(C[0][3], C[1][2]));
    double2 r = make_double2(0.0, 0.0);
    if (lane == 0) {
        auto& A = st.C;
        for (int i = 0; i < m2; i++) {
            A[i][i] = make_double2(0.0, 0.0);
            for (int j = 0; j < i; j++) A[i][j] = make_double2(-A[j][i].x, -A[j][i].y);
        }
        double2 pf = make_double2(1.0, 0.0);
        for (int k = 0; k < m2 - 1; k += 2) {
            int kp = k + 1;
            double best = zabs2(A[k + 1][k]);
            for (int i = k + 2; i < m2; i++)
                if (zabs2(A[i][k]) > best) {
                    best = zabs2(A[i][k]);
                    kp = i;
                }
            if (kp != k + 1) {
                for (int c = 0; c < m2; c++) {
                    const double2 t = A[k + 1][c];
                    A[k + 1][c] = A[kp][c];
                    A[kp][c] = t;
                }
                for (int q = 0; q < m2; q++) {
                    const double2 t = A[q][k + 1];
                    A[q][k + 1] = A[q][kp];
                    A[q][kp] = t;
                }
                pf = make_double2(-pf.x, -pf.y);
            }
            const double2 piv = A[k][k + 1];
            pf = zmul(pf, piv);
            if (piv.x == 0.0 && piv.y == 0.0) break;
            const double2 ip = zrcp(piv);
            for (int i = k + 2; i < m2; i++) {
                const double2 ti = zmul(A[k][i], ip);
                for (int j = k + 2; j < m2; j++) {
                    const double2 tj = zmul(A[k][j], ip);
                    A[i][j] = zadd(A[i][j], zsub(zmul(ti, A[j][k + 1]), zmul(A[i][k + 1], tj)));
                }
            }
        }
        r = pf;
    }
    return zshfl(r, 0);
}

// psi ratio factor of the Pfaffian for flipping sites fl[0..nf) (nf <= 4) of
// configuration `bits` (pfaffian::psi_over_psi via update_context).  Xi(t)
// returns X^{-1}[lane][t] (t a compile-time index when unrolled), Xcol(f)
// returns X^{-1}[lane][f] for a runtime f.  Leaves X^{-1}B in st.IB and in
// ib (this lane's row) and C^{-1} in st.C for pf_accept.  Warp-collective.
template <int NF, typename XI, typename XCOL>
__device__ __forceinline__ double2 pf_ratio(const PfDev& p, uint32_t bits, const int* fl, int lane, PfStage& st,
                                            XI Xi, XCOL Xcol, double2 (&ib)[2 * kPfMaxFlips]) {
    static_assert(NF >= 1 && NF <= kPfMaxFlips, "1..4 flips");
    constexpr int nf = NF;
    const int n = p.n;
    uint32_t fm = 0;
#pragma unroll
    for (int q = 0; q < nf; q++) fm |= 1u << fl[q];
    // B: dense columns k < nf (the unit columns nf + k are implicit)
#pragma unroll
    for (int k = 0; k < nf; k++) {
        double2 b = make_double2(0.0, 0.0);
        if (lane < n && lane != fl[k]) {
            const double2 a1 = pf_elem(p, bits, lane, fl[k], (fm >> lane) & 1u, 1);
            const double2 a0 = pf_elem(p, bits, lane, fl[k], 0, 0);
            b = zsub(a1, a0);
        }
        st.B[lane][k] = b;
    }
    __syncwarp();
    // this lane's row of X^{-1} B
#pragma unroll
    for (int k = 0; k < nf; k++) {
        double2 a0 = make_double2(0.0, 0.0), a1 = a0;
#pragma unroll
        for (int t = 0; t < kPfMaxSites; t += 2) {
            a0 = zfma(Xi(t), st.B[t][k], a0);
            a1 = zfma(Xi(t + 1), st.B[t + 1][k], a1);
        }
        ib[k] = zadd(a0, a1);
        ib[nf + k] = Xcol(fl[k]);
    }
#pragma unroll
    for (int q = 0; q < 2 * nf; q++) st.IB[lane][q] = ib[q];
    __syncwarp();
    // C^{-1}[r][q], r < q: one pair per lane
    const int m2 = 2 * nf;
    const int npairs = m2 * (m2 - 1) / 2;
    if (lane < npairs) {
        int r = 0, q = lane;
        while (q >= m2 - 1 - r) {
            q -= m2 - 1 - r;
            r++;
        }
        q += r + 1;
        // (tmp - tmp^T)[r][q] = 1/2 sum_t (B[t][r] IB[t][q] - B[t][q] IB[t][r])
        double2 acc = make_double2(0.0, 0.0);
        if (r < nf) {
            for (int t = 0; t < n; t++) acc = zfma(st.B[t][r], st.IB[t][q], acc);
        } else {
            acc = zadd(acc, st.IB[fl[r - nf]][q]);
        }
        if (q < nf) {
            for (int t = 0; t < n; t++) acc = zsub(acc, zmul(st.B[t][q], st.IB[t][r]));
        } else {
            acc = zsub(acc, st.IB[fl[q - nf]][r]);
        }
        acc = zscale(acc, 0.5);
        // C0: C(nf + k, k) = 1 and C(k, l) = a(f_k, f_l) - a'(f_k, f_l), l < k
        if (r < nf && q == nf + r) acc.x -= 1.0;
        if (q < nf) {
            const double2 d = zsub(pf_elem(p, bits, fl[q], fl[r], 0, 0), pf_elem(p, bits, fl[q], fl[r], 1, 1));
            acc = zsub(acc, d);
        }
        st.C[r][q] = acc;
    }
    __syncwarp();
    const double2 pf = pf_small(st, m2, lane);
    const int sgn = ((nf * (nf + 1) / 2) & 1) ? -1 : 1;
    return sgn > 0 ? pf : make_double2(-pf.x, -pf.y);
}

// X^{-1} update after an accepted move of nf <= 2 flips (pfaffian.cpp:360-386):
// with Ca = (C^{-1})^{-1} (antisymmetric), X^{-1} += (X^{-1}B) Ca (X^{-1}B)^T,
// which equals the reference's T2 - T2^T with T2 = X^{-1}B Ca (X^{-1}B)^T / 2.
// Uses st.C / st.IB / ib from the pf_ratio call of the same proposal; lane i
// updates row i of A.
__device__ __forceinline__ void pf_accept(int nf, int lane, const PfStage& st, const double2 (&ib)[2 * kPfMaxFlips],
                                          double2* A, int n) {
    double2 Ca[4][4];
    const auto& C = st.C;
    if (nf == 1) {
        const double2 ic = zrcp(C[0][1]);
        Ca[0][0] = Ca[1][1] = make_double2(0.0, 0.0);
        Ca[0][1] = make_double2(-ic.x, -ic.y);
        Ca[1][0] = ic;
    } else {
        const double2 c01 = C[0][1], c02 = C[0][2], c03 = C[0][3], c12 = C[1][2], c13 = C[1][3], c23 = C[2][3];
        const double2 ip = zrcp(zadd(zsub(zmul(c01, c23), zmul(c02, c13)), zmul(c03, c12)));
        auto s = [&](double2 v, double sg) { const double2 w = zmul(v, ip); return make_double2(sg * w.x, sg * w.y); };
        Ca[0][0] = Ca[1][1] = Ca[2][2] = Ca[3][3] = make_double2(0.0, 0.0);
        Ca[0][1] = s(c23, -1.0); Ca[0][2] = s(c13, 1.0); Ca[0][3] = s(c12, -1.0);
        Ca[1][0] = s(c23, 1.0); Ca[1][2] = s(c03, -1.0); Ca[1][3] = s(c02, 1.0);
        Ca[2][0] = s(c13, -1.0); Ca[2][1] = s(c03, 1.0); Ca[2][3] = s(c01, -1.0);
        Ca[3][0] = s(c12, 1.0); Ca[3][1] = s(c02, -1.0); Ca[3][2] = s(c01, 1.0);
    }
    const int m2 = 2 * nf;
    double2 t1[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int t = 0; t < 4; t++)
            if (t < m2 && q < m2) acc = zfma(ib[t], Ca[t][q], acc);
        t1[q] = acc;
    }
    if (lane < n) {
        for (int j = 0; j < n; j++) {
            double2 acc = A[lane * kPfLd + j];
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (q < m2) acc = zfma(t1[q], st.IB[j][q], acc);
            A[lane * kPfLd + j] = acc;
        }
    }
    __syncwarp();
}

// log Pf(X) of configuration `bits` (pfaffian.cpp:294-296, PFAPACK skpf10
// 'P' pivoting): Parlett-Reid tridiagonalisation on the warp's smem copy A
// (leading dimension kPfLd), lane = row.  Returns log|Pf| + i arg(Pf) on
// every lane (modulo 2 pi i); -inf real part for a singular X.
__device__ __forceinline__ double2 pf_log_pfaffian(const PfDev& p, uint32_t bits, int lane, double2* A) {
    const int n = p.n;
    if (lane < n)
        for (int j = 0; j < n; j++) A[lane * kPfLd + j] = pf_elem(p, bits, lane, j, 0, 0);
    __syncwarp();
    double lre = 0.0, lim = 0.0;
    int swaps = 0;
    bool zero = (n & 1) != 0;
    for (int k = 0; k + 1 < n && !zero; k += 2) {
        const bool cand = lane >= k + 1 && lane < n;
        const int kp = warp_argmax(cand ? zabs2(A[lane * kPfLd + k]) : -1.0);
        if (kp != k + 1) {
            if (lane < n) {  // swap rows k+1, kp (lane = column), then columns
                const double2 t = A[(k + 1) * kPfLd + lane];
                A[(k + 1) * kPfLd + lane] = A[kp * kPfLd + lane];
                A[kp * kPfLd + lane] = t;
            }
            __syncwarp();
            if (lane < n) {
                const double2 t = A[lane * kPfLd + k + 1];
                A[lane * kPfLd + k + 1] = A[lane * kPfLd + kp];
                A[lane * kPfLd + kp] = t;
            }
            __syncwarp();
            swaps++;
        }
        const double2 piv = A[k * kPfLd + k + 1];
        const double2 sub = A[(k + 1) * kPfLd + k];
        if (sub.x == 0.0 && sub.y == 0.0) {
            zero = true;
            break;
        }
        lre += 0.5 * log(zabs2(piv));
        lim += atan2(piv.y, piv.x);
        if (k + 2 < n) {
            const double2 ip = zrcp(piv);
            if (lane >= k + 2 && lane < n) {
                const double2 ti = zmul(A[k * kPfLd + lane], ip);
                const double2 ai = A[lane * kPfLd + k + 1];
                for (int j = k + 2; j < n; j++) {
                    const double2 tj = zmul(A[k * kPfLd + j], ip);
                    const double2 upd = zsub(zmul(ti, A[j * kPfLd + k + 1]), zmul(ai, tj));
                    A[lane * kPfLd + j] = zadd(A[lane * kPfLd + j], upd);
                }
            }
        }
        __syncwarp();
    }
    if (zero) return make_double2(-INFINITY, 0.0);
    return make_double2(lre, lim + (swaps & 1 ? 3.14159265358979323846 : 0.0));
}

// Pfaffian part of O_k (pfaffian.cpp:399-415) from the antisymmetric X^{-1}
// in the warp's smem matrix A (leading dimension kPfLd); deterministic
// gather per class.
template <typename TO>
__device__ __forceinline__ void pf_derivative(const PfDev& p, uint32_t bits, int lane, const double2* A, TO* out) {
    for (int a = lane; a < p.n_indep; a += 32) {
        double2 acc[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
        for (int e = p.pair_ptr[a]; e < p.pair_ptr[a + 1]; e++) {
            const uint32_t w = p.pairs[e];
            const int i = w >> 16, j = (w >> 8) & 0xff, pos = w & 1;
            const double2 v = A[i * kPfLd + j];
            const int sp = (((bits >> i) & 1) << 1) + ((bits >> j) & 1);
            acc[sp] = pos ? zsub(acc[sp], v) : zadd(acc[sp], v);
        }
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if constexpr (sizeof(TO) == 16)
                out[a + p.n_indep * c] = acc[c];
            else
                out[a + p.n_indep * c] = make_float2((float)acc[c].x, (float)acc[c].y);
        }
    }
}

// ---------------------------------------------------------------------------
// Sweep form.  The Metropolis sweep keeps X^{-1} (antisymmetric) as its
// circulant half, Cx[(d - 1) * 32 + i] = X^{-1}[i][(i + d) & 31] for
// d = 1..16: 8 KB per warp instead of the 16.9 KB square, so that a block
// holds about twice the chains.  Lane i walks its row in offset order (the
// entries (i, i + d) from Cx[d][i], the entries (i, i - d) as -Cx[d][i - d]),
// both conflict-free across the warp.  The pair (i, i + 16) is held twice,
// once per orientation, and each copy is updated by its own row's formula.
// Rows and columns >= n are zero and stay zero.
constexpr int kPfCircBytes = 16 * kPfMaxSites * 16;
constexpr int kPfSweepFlips = 2;  // sweep proposals: one spin or one bond

struct PfSweepStage {
    double2 BT[kPfSweepFlips][kPfMaxSites];      // dense columns of B, column-major
    double2 IB[2 * kPfSweepFlips][kPfMaxSites];  // X^{-1} B, column-major
    int piv[kPfMaxSites];                        // Gauss-Jordan pivot row of each column
    int qinv[kPfMaxSites];                       // inverse of piv
};

// X^{-1}[i][j] from the circulant half (branch-free: the entries (i, i + d),
// d <= 16, are held by row i, the others as -X^{-1}[j][i] by row j)
__device__ __forceinline__ double2 pf_circ_at(const double2* Cx, int i, int j) {
    const int d = (j - i) & 31;
    const bool fw = d <= 16;
    const double2 v = Cx[d == 0 ? 0 : (fw ? (d - 1) * kPfMaxSites + i : (31 - d) * kPfMaxSites + j)];
    const double s = d == 0 ? 0.0 : (fw ? 1.0 : -1.0);
    return make_double2(s * v.x, s * v.y);
}

// Unscramble and antisymmetrise the Gauss-Jordan result A (leading dimension
// LD) into the circulant half: Cx(i, j) = (X^{-1}[i][j] - X^{-1}[j][i]) / 2
// with X^{-1}[k][m] = A[piv[k]][qinv[m]].
template <int LD>
__device__ __forceinline__ void pf_unscramble_circ(int n, int lane, const double2* A, const PfSweepStage& st,
                                                   double2* Cx) {
    const int pi = lane < n ? st.piv[lane] : 0, qi = lane < n ? st.qinv[lane] : 0;
#pragma unroll 4
    for (int d = 1; d <= 16; d++) {
        const int j = (lane + d) & 31;
        double2 v = make_double2(0.0, 0.0);
        if (lane < n && j < n) {
            const double2 a = A[pi * LD + st.qinv[j]], b = A[st.piv[j] * LD + qi];
            v = make_double2(0.5 * (a.x - b.x), 0.5 * (a.y - b.y));
        }
        Cx[(d - 1) * kPfMaxSites + lane] = v;
    }
}

// Fresh context in circulant form: Gauss-Jordan in the warp's global
// scratch gscr (leading dimension 32; it stays in L1, which a square
// workspace in shared memory would shrink for every warp of the block), then
// X^{-1} unscrambled and antisymmetrised straight into Cx:
// Cx(i, j) = (X^{-1}[i][j] - X^{-1}[j][i]) / 2 with X^{-1}[k][m] =
// A[piv[k]][qinv[m]] (pfaffian.cpp:284-297).  Warp-collective.
__device__ __forceinline__ void pf_fresh_circ(const PfDev& p, uint32_t bits, int lane, double2* Cx, PfSweepStage& st,
                                              double2* gscr) {
    const int n = p.n;
    pf_gauss_jordan<kPfMaxSites>(p, bits, lane, gscr, st.piv, &st.BT[0][0]);
    if (lane < n) st.qinv[st.piv[lane]] = lane;
    __syncwarp();
    pf_unscramble_circ<kPfMaxSites>(n, lane, gscr, st, Cx);
    __syncwarp();
}

// Butterfly warp sum of a complex value (every lane gets the same result:
// IEEE addition is commutative).
__device__ __forceinline__ double2 zwarp_sum(double2 v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
    }
    return v;
}

// Pairs of the 2 NF x 2 NF matrix C^{-1} (r < q), every lane: NF = 1: c[0]
// = (0, 1); NF = 2: c = (0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3).
template <int NF> struct PfPairs {
    double2 c[NF == 1 ? 1 : 6];
};

// psi ratio factor of the Pfaffian for flipping sites fl[0..NF) with X^{-1}
// in circulant form (the same rank-2m formula as pf_ratio).  Lane t holds
// row t of B and of X^{-1} B (ib), so each entry of C^{-1} is one warp sum
// of lane products plus entries of X^{-1} B on the flipped sites' lanes.
// Leaves X^{-1} B in st.IB (and this lane's row in ib) and C^{-1} in cp for
// pf_accept_circ.  Warp-collective.
template <int NF>
__device__ __forceinline__ double2 pf_ratio_circ(const PfDev& p, uint32_t bits, const int* fl, int lane,
                                                 PfSweepStage& st, const double2* Cx, double2 (&ib)[2 * NF],
                                                 PfPairs<NF>& cp) {
    static_assert(NF == 1 || NF == 2, "sweep proposals flip one or two sites");
    const int n = p.n;
    uint32_t fm = 0;
#pragma unroll
    for (int q = 0; q < NF; q++) fm |= 1u << fl[q];
    double2 b[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
        b[k] = make_double2(0.0, 0.0);
        if (lane < n && lane != fl[k]) {
            const double2 a1 = pf_elem(p, bits, lane, fl[k], (fm >> lane) & 1u, 1);
            const double2 a0 = pf_elem(p, bits, lane, fl[k], 0, 0);
            b[k] = zsub(a1, a0);
        }
        st.BT[k][lane] = b[k];
    }
    __syncwarp();
    // this lane's row of X^{-1} B: the entries (i, i + d) and (i, i - d)
    double2 up[NF], dn[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) up[k] = dn[k] = make_double2(0.0, 0.0);
#pragma unroll 4
    for (int d = 1; d <= 16; d++) {
        const int j = (lane + d) & 31;
        const double2 x = Cx[(d - 1) * kPfMaxSites + lane];
#pragma unroll
        for (int k = 0; k < NF; k++) up[k] = zfma(x, st.BT[k][j], up[k]);
    }
#pragma unroll 5
    for (int d = 1; d <= 15; d++) {
        const int j = (lane - d) & 31;
        const double2 x = Cx[(d - 1) * kPfMaxSites + j];
#pragma unroll
        for (int k = 0; k < NF; k++) dn[k] = zfma(x, st.BT[k][j], dn[k]);
    }
#pragma unroll
    for (int k = 0; k < NF; k++) {
        ib[k] = zsub(up[k], dn[k]);
        ib[NF + k] = pf_circ_at(Cx, lane, fl[k]);
    }
#pragma unroll
    for (int q = 0; q < 2 * NF; q++) st.IB[q][lane] = ib[q];
    // X^{-1} B entries on the flipped sites' lanes
    auto at = [&](int q, int site) { return zshfl(ib[q], site); };
    if constexpr (NF == 1) {
        // (0, 1): (sum_t B_t0 IB_t1 - IB_{f0,0}) / 2 - 1
        const double2 s = zwarp_sum(zmul(b[0], ib[1]));
        double2 c = zscale(zsub(s, at(0, fl[0])), 0.5);
        c.x -= 1.0;
        cp.c[0] = c;
        return make_double2(-c.x, -c.y);  // (-1)^{m(m+1)/2}, m = 1
    } else {
        const double2 s01 = zwarp_sum(zsub(zmul(b[0], ib[1]), zmul(b[1], ib[0])));
        const double2 s02 = zwarp_sum(zmul(b[0], ib[2]));
        const double2 s03 = zwarp_sum(zmul(b[0], ib[3]));
        const double2 s12 = zwarp_sum(zmul(b[1], ib[2]));
        const double2 s13 = zwarp_sum(zmul(b[1], ib[3]));
        const double2 i00 = at(0, fl[0]), i01 = at(1, fl[0]), i03 = at(3, fl[0]);
        const double2 i10 = at(0, fl[1]), i11 = at(1, fl[1]), i12 = at(2, fl[1]);
        // C0: C(k, l) = a(f_k, f_l) - a'(f_k, f_l) below the diagonal block
        const double2 d01 = zsub(pf_elem(p, bits, fl[1], fl[0], 0, 0), pf_elem(p, bits, fl[1], fl[0], 1, 1));
        cp.c[0] = zsub(zscale(s01, 0.5), d01);
        cp.c[1] = zscale(zsub(s02, i00), 0.5);
        cp.c[1].x -= 1.0;
        cp.c[2] = zscale(zsub(s03, i10), 0.5);
        cp.c[3] = zscale(zsub(s12, i01), 0.5);
        cp.c[4] = zscale(zsub(s13, i11), 0.5);
        cp.c[4].x -= 1.0;
        cp.c[5] = zscale(zsub(i03, i12), 0.5);
        const double2 pf = zadd(zsub(zmul(cp.c[0], cp.c[5]), zmul(cp.c[1], cp.c[4])), zmul(cp.c[2], cp.c[3]));
        return make_double2(-pf.x, -pf.y);  // (-1)^{m(m+1)/2}, m = 2
    }
}

// X^{-1} update after an accepted move (pf_accept in circulant form): with
// Ca = (C^{-1})^{-1}, t1 = (row i of X^{-1} B) Ca and
// X^{-1}(i, i + d) += t1 . (row i + d of X^{-1} B), d = 1..16.
template <int NF>
__device__ __forceinline__ void pf_accept_circ(int lane, const PfSweepStage& st, const double2 (&ib)[2 * NF],
                                               const PfPairs<NF>& cp, double2* Cx, int n) {
    double2 t1[2 * NF];
    if constexpr (NF == 1) {
        // Ca = [[0, -1/c], [1/c, 0]]
        const double2 ic = zrcp(cp.c[0]);
        t1[0] = zmul(ib[1], ic);
        t1[1] = zmul(ib[0], make_double2(-ic.x, -ic.y));
    } else {
        const double2 c01 = cp.c[0], c02 = cp.c[1], c03 = cp.c[2], c12 = cp.c[3], c13 = cp.c[4], c23 = cp.c[5];
        const double2 ip = zrcp(zadd(zsub(zmul(c01, c23), zmul(c02, c13)), zmul(c03, c12)));
        // Ca = adj / Pf: Ca[t][q] for t != q (antisymmetric)
        const double2 a01 = zmul(c23, ip), a02 = zmul(c13, ip), a03 = zmul(c12, ip);
        const double2 a12 = zmul(c03, ip), a13 = zmul(c02, ip), a23 = zmul(c01, ip);
        // Ca[0][1] = -a01, Ca[0][2] = a02, Ca[0][3] = -a03, Ca[1][2] = -a12,
        // Ca[1][3] = a13, Ca[2][3] = -a23; Ca[q][t] = -Ca[t][q]
        // t1[q] = sum_t ib[t] Ca[t][q]
        t1[0] = zsub(zsub(zmul(ib[1], a01), zmul(ib[2], a02)), zmul(ib[3], make_double2(-a03.x, -a03.y)));
        t1[1] = zsub(zadd(zmul(ib[0], make_double2(-a01.x, -a01.y)), zmul(ib[2], a12)), zmul(ib[3], a13));
        t1[2] = zadd(zadd(zmul(ib[0], a02), zmul(ib[1], make_double2(-a12.x, -a12.y))), zmul(ib[3], a23));
        t1[3] = zadd(zadd(zmul(ib[0], make_double2(-a03.x, -a03.y)), zmul(ib[1], a13)),
                     zmul(ib[2], make_double2(-a23.x, -a23.y)));
    }
    __syncwarp();  // st.IB of every lane
    if (lane < n) {
#pragma unroll 4
        for (int d = 1; d <= 16; d++) {
            const int j = (lane + d) & 31;
            double2 acc = Cx[(d - 1) * kPfMaxSites + lane];
#pragma unroll
            for (int q = 0; q < 2 * NF; q++) acc = zfma(t1[q], st.IB[q][j], acc);
            Cx[(d - 1) * kPfMaxSites + lane] = acc;
        }
    }
    __syncwarp();
}

}  // namespace rbmnqs
