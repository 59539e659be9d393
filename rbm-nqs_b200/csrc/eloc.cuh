// eloc.cuh -- evaluation kernel of the FP32 hot path: local energy
// E_loc = sum_ops sum_l' H[l, l'] psi(sigma_l') / psi(sigma) (local_op.cpp:31-60)
// and log-derivatives O_k (rbm_base.cpp:194-217, rbm_symmetry.cpp:97-130) of
// every sampled configuration, one warp per configuration.
//
// Layout.  theta (T = nh S entries, t = k + nh s) is split into groups of KB
// consecutive hidden units k with the same symmetry index s; lane l owns
// groups g = l + 32 j (j < NG), so E = KB NG entries per lane.  Flipping site
// f adds -2 sigma_f W[P_s(f), k0 .. k0 + KB - 1] to a group: one byte of the
// symmetry table and one KB x 8-byte row segment of W per group, read from
// shared memory (rows padded to an odd number of 16-byte units, so the lanes'
// random rows spread over the banks).
//
// E_loc.  The Hamiltonian comes as a table of terms (operator, flip mask,
// value per local configuration; TermDev).  For each term the lanes form
// theta' of their entries and the grouped FP32 ln cosh sum (lnc_lane: one
// ex2, sin and cos per entry, one lg2 and rsqrt per four), giving a partial
// log magnitude and unit phase of psi'/psi.  KT terms at a time, the partials
// are reduced with a butterfly that leaves term q on lanes with
// (lane >> (5 - log2 KT)) == q, so the remaining per-term work (bias, exp and
// rotation, the matrix element, accumulation) runs once per term on
// different lanes instead of once per term on every lane.
//
// theta itself is recomputed in FP64 from the all-up table (hb + sum_f W)
// minus 2 W over the down spins; tanh theta (for O_k) is evaluated in FP64
// and stored as FP32 in the warp's scratch.
#pragma once

#include "common.cuh"
#include "sampler.cuh"

namespace rbmnqs {
namespace eloc {

// Warps per block and resident blocks per SM by entries per lane: up to 4
// entries, 8-warp blocks at up to 85 registers (3 blocks, 24 warps per SM);
// above, 16-warp blocks at up to 128 registers.
__host__ __device__ constexpr int eloc_warps(int E) { return E <= 4 ? 8 : 16; }
__host__ __device__ constexpr int eloc_min_blocks(int E) { return E <= 4 ? 3 : 1; }

__host__ __device__ inline int a16(int x) { return (x + 15) & ~15; }

// Row stride of the padded FP32 W copy in shared memory, in float2: an odd
// number of 16-byte units when rows are read 16 or 32 bytes at a time.
__host__ __device__ inline int w32_stride(int nh, int kb) {
    if (kb == 1) return nh;
    int u = (nh * 8 + 15) / 16;
    if ((u & 1) == 0) u++;
    return 2 * u;
}

// Shared-memory carve-up, the same arithmetic on host (sizing) and device.
struct ElocLayout {
    int w32, w64, perm, inv, base, terms, diag, vals, vb, warp0, warp_bytes, total;
    int wstride;                      // row stride of the W32 the kernel reads (float2)
    int w32_smem, w64_smem, vals_smem, inv_smem;
};

__host__ __device__ inline ElocLayout eloc_layout(const MachineDev& m, const TermTable& tt, int kb, int warps,
                                                  bool with_O, int budget) {
    ElocLayout L{};
    const int ws = w32_stride(m.nh, kb);
    int off = 0;
    L.warp_bytes = a16(16 + m.T * 8);
    // fixed parts first: warps' scratch, base theta, symmetry table, terms, bias
    const int warps_b = warps * L.warp_bytes;
    const int base_b = a16(m.T * 16);
    const int perm_b = m.symmetric ? a16(m.n * m.S) : 0;
    const int terms_b = a16((tt.n_terms + tt.n_diag) * (int)sizeof(TermDev));
    const int vb_b = a16(m.n_vb * 16);
    int need = warps_b + base_b + perm_b + terms_b + vb_b;
    const int w32_b = a16(m.n * ws * 8), vals_b = a16(tt.n_vals * 16), w64_b = a16(m.n * m.nh * 16);
    const int inv_b = (m.symmetric && with_O) ? a16(m.n * m.S) : 0;
    // optional parts in order of use per configuration
    L.w32_smem = need + w32_b <= budget;
    if (L.w32_smem) need += w32_b;
    L.vals_smem = need + vals_b <= budget;
    if (L.vals_smem) need += vals_b;
    L.inv_smem = inv_b > 0 && need + inv_b <= budget;
    if (L.inv_smem) need += inv_b;
    L.w64_smem = need + w64_b <= budget;
    if (L.w64_smem) need += w64_b;
    L.wstride = L.w32_smem ? ws : m.nh;
    L.w32 = off;
    off += L.w32_smem ? w32_b : 0;
    L.w64 = off;
    off += L.w64_smem ? w64_b : 0;
    L.perm = off;
    off += perm_b;
    L.inv = off;
    off += L.inv_smem ? inv_b : 0;
    L.base = off;
    off += base_b;
    L.terms = off;
    L.diag = off + tt.n_terms * (int)sizeof(TermDev);
    off += terms_b;
    L.vals = off;
    off += L.vals_smem ? vals_b : 0;
    L.vb = off;
    off += vb_b;
    L.warp0 = off;
    off += warps_b;
    L.total = off;
    return L;
}

__device__ __forceinline__ int sbit(const uint32_t (&sp)[4], int i) {
    const uint32_t w = i < 32 ? sp[0] : (i < 64 ? sp[1] : (i < 96 ? sp[2] : sp[3]));
    return (w >> (i & 31)) & 1;
}
__device__ __forceinline__ int byte_of(uint32_t w, int q) { return (w >> (8 * q)) & 0xff; }
__device__ __forceinline__ int term_flip(const TermDev& t, int q) { return q < 4 ? byte_of(t.flip0, q) : byte_of(t.flip1, q - 4); }
__device__ __forceinline__ int term_site(const TermDev& t, int q) { return q < 4 ? byte_of(t.site0, q) : byte_of(t.site1, q - 4); }
__device__ __forceinline__ int term_nf(const TermDev& t) { return byte_of(t.flip1, 2); }
__device__ __forceinline__ int term_k(const TermDev& t) { return byte_of(t.flip1, 3); }

__device__ __forceinline__ int term_loc(const TermDev& t, const uint32_t (&sp)[4]) {
    const int k = term_k(t);
    int loc = 0;
    for (int i = 0; i < k; i++) loc |= sbit(sp, term_site(t, i)) << i;
    return loc;
}

// visible-bias index f mod n_vb (rbm_base.cpp:310)
__device__ __forceinline__ int vbi(int f, int n_vb, int n) {
    return n_vb == n ? f : ((n_vb & (n_vb - 1)) == 0 ? (f & (n_vb - 1)) : f % n_vb);
}

template <int KB> struct Row;
template <> struct Row<1> {
    static __device__ __forceinline__ void ld(const float2* p, float2 (&w)[1]) { w[0] = *p; }
};
template <> struct Row<2> {
    static __device__ __forceinline__ void ld(const float2* p, float2 (&w)[2]) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        w[0] = make_float2(v.x, v.y);
        w[1] = make_float2(v.z, v.w);
    }
};
template <> struct Row<4> {
    static __device__ __forceinline__ void ld(const float2* p, float2 (&w)[4]) {
        const float4 v0 = reinterpret_cast<const float4*>(p)[0];
        const float4 v1 = reinterpret_cast<const float4*>(p)[1];
        w[0] = make_float2(v0.x, v0.y);
        w[1] = make_float2(v0.z, v0.w);
        w[2] = make_float2(v1.x, v1.y);
        w[3] = make_float2(v1.z, v1.w);
    }
};

// Butterfly reduce-scatter of KT per-lane partials (log magnitude summed,
// unit phase multiplied): afterwards every lane holds the total of term
// (lane >> (5 - log2 KT)), the same on the 32 / KT lanes of that term.
template <int KT>
__device__ __forceinline__ void reduce_terms(float (&re)[KT], float2 (&u)[KT], int lane, float& R, float2& U) {
    static_assert(KT == 4 || KT == 8, "4 or 8 terms per round");
#pragma unroll
    for (int stage = 0; stage < (KT == 8 ? 3 : 2); stage++) {
        const int off = 16 >> stage;
        const int cnt = KT >> stage, half = cnt >> 1;
        const bool up = (lane & off) != 0;
#pragma unroll
        for (int i = 0; i < KT / 2; i++) {
            if (i >= half) break;
            const float kr = up ? re[half + i] : re[i], sr = up ? re[i] : re[half + i];
            const float2 ku = up ? u[half + i] : u[i], su = up ? u[i] : u[half + i];
            const float rr = __shfl_xor_sync(kFull, sr, off);
            float2 ru;
            ru.x = __shfl_xor_sync(kFull, su.x, off);
            ru.y = __shfl_xor_sync(kFull, su.y, off);
            re[i] = kr + rr;
            u[i] = cmul(ku, ru);
        }
    }
    float r = re[0];
    float2 v = u[0];
#pragma unroll
    for (int off = (KT == 8 ? 2 : 4); off >= 1; off >>= 1) {
        r += __shfl_xor_sync(kFull, r, off);
        float2 w;
        w.x = __shfl_xor_sync(kFull, v.x, off);
        w.y = __shfl_xor_sync(kFull, v.y, off);
        v = cmul(v, w);
    }
    R = r;
    U = v;
}

template <int KB, int NG, bool SYM, int NFM>
__global__ void __launch_bounds__(32 * eloc_warps(KB* NG), eloc_min_blocks(KB* NG))
    eloc_kernel(const EvalArgs a, const ElocLayout L) {
    constexpr int E = KB * NG;
    constexpr int WARPS = eloc_warps(E);
    constexpr int KT = E >= 16 ? 4 : 8;  // terms per reduction round
    extern __shared__ __align__(16) unsigned char smem[];
    const MachineDev& m = a.m;
    const int n = m.n, nh = m.nh, S = m.S, T = m.T, n_vb = m.n_vb;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int n_terms = a.tt.n_terms, n_diag = a.tt.n_diag;

    // ---- block tables
    float2* sW32 = reinterpret_cast<float2*>(smem + L.w32);
    double2* sW64 = reinterpret_cast<double2*>(smem + L.w64);
    uint8_t* sPerm = smem + L.perm;
    uint8_t* sInv = smem + L.inv;
    double2* sBase = reinterpret_cast<double2*>(smem + L.base);
    TermDev* sTerms = reinterpret_cast<TermDev*>(smem + L.terms);
    TermDev* sDiag = reinterpret_cast<TermDev*>(smem + L.diag);
    double2* sVals = reinterpret_cast<double2*>(smem + L.vals);
    double2* sVb = reinterpret_cast<double2*>(smem + L.vb);
    if (L.w32_smem)
        for (int i = tid; i < n * nh; i += nthr) sW32[(i / nh) * L.wstride + i % nh] = m.W32[i];
    if (L.w64_smem)
        for (int i = tid; i < n * nh; i += nthr) sW64[i] = m.W64[i];
    if (SYM) {
        for (int i = tid; i < n * S; i += nthr) sPerm[i] = m.perm[i];
        if (L.inv_smem)
            for (int i = tid; i < n * S; i += nthr) sInv[i] = m.inv[i];
    }
    for (int i = tid; i < n_terms; i += nthr) sTerms[i] = a.tt.terms[i];
    for (int i = tid; i < n_diag; i += nthr) sDiag[i] = a.tt.diag[i];
    if (L.vals_smem)
        for (int i = tid; i < a.tt.n_vals; i += nthr) sVals[i] = a.tt.vals[i];
    for (int i = tid; i < n_vb; i += nthr) sVb[i] = m.vb[i];
    __syncthreads();
    const float2* W32 = L.w32_smem ? sW32 : m.W32;
    const double2* W64 = L.w64_smem ? sW64 : m.W64;
    const uint8_t* inv = L.inv_smem ? sInv : m.inv;
    const double2* vals = L.vals_smem ? sVals : a.tt.vals;
    const int ws = L.wstride;
    // theta of the all-up configuration (FP64): hb_k + sum_f W[P_s(f), k]
    for (int t = tid; t < T; t += nthr) {
        const int k = t % nh, s = t / nh;
        double2 acc = m.hb[k];
        for (int f = 0; f < n; f++) {
            const double2 w = W64[(SYM ? (int)sPerm[f * S + s] : f) * nh + k];
            acc.x += w.x;
            acc.y += w.y;
        }
        sBase[t] = acc;
    }
    __syncthreads();

    const int warp = tid >> 5, lane = tid & 31;
    unsigned char* wbase = smem + L.warp0 + warp * L.warp_bytes;
    float2* tn = reinterpret_cast<float2*>(wbase + 16);
    // the lane's groups: symmetry index s, first hidden unit k0, validity
    const int G = T / KB, NGK = nh / KB;
    int gs[NG], gk[NG];
    uint32_t vmask = 0;
#pragma unroll
    for (int j = 0; j < NG; j++) {
        const int g = lane + 32 * j;
        const bool ok = g < G;
        gs[j] = ok ? g / NGK : 0;
        gk[j] = ok ? (g % NGK) * KB : 0;
        vmask |= ok ? 1u << j : 0u;
    }
    const int nv = KB * __popc(vmask);

    for (int b = blockIdx.x * WARPS + warp; b < a.B; b += gridDim.x * WARPS) {
        uint32_t sp[4];
#pragma unroll
        for (int w = 0; w < 4; w++) sp[w] = a.spins[4 * b + w];

        // ---- theta in FP64 (down spins subtracted from the all-up table),
        // rounded to FP32; tanh theta in FP64 into the warp's scratch
        float2 th[E];
#pragma unroll
        for (int j = 0; j < NG; j++) {
            double2 acc[KB];
            const bool ok = (vmask >> j) & 1u;
            const int t0 = gk[j] + nh * gs[j];
#pragma unroll
            for (int i = 0; i < KB; i++) acc[i] = ok ? sBase[t0 + i] : make_double2(0, 0);
            if (ok) {
#pragma unroll
                for (int wd = 0; wd < 4; wd++) {
                    uint32_t bits = sp[wd];
                    while (bits) {
                        const int f = 32 * wd + __ffs(bits) - 1;
                        bits &= bits - 1;
                        const int row = SYM ? (int)sPerm[f * S + gs[j]] : f;
                        const double2* wr = W64 + row * nh + gk[j];
#pragma unroll
                        for (int i = 0; i < KB; i++) {
                            const double2 w = wr[i];
                            acc[i].x = fma(-2.0, w.x, acc[i].x);
                            acc[i].y = fma(-2.0, w.y, acc[i].y);
                        }
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < KB; i++) {
                th[j * KB + i] = make_float2((float)acc[i].x, (float)acc[i].y);
                if (ok && a.O) {
                    const C2<double> tt = ctanh_r<double>(acc[i].x, acc[i].y);
                    tn[t0 + i] = make_float2((float)tt.x, (float)tt.y);
                }
            }
        }

        double ex = 0.0, ey = 0.0;
        if (a.eloc) {
            // diagonal matrix elements, one operator per lane
            for (int d = lane; d < n_diag; d += 32) {
                const TermDev td = sDiag[d];
                const double2 v = vals[td.voff + term_loc(td, sp)];
                ex += v.x;
                ey += v.y;
            }
            // ln cosh sum of the current theta
            float cre;
            float2 cu;
            lnc_lane<E>(th, nv, cre, cu);
            // off-diagonal terms, KT per round
            for (int c0 = 0; c0 < n_terms; c0 += KT) {
                float pre[KT];
                float2 pu[KT];
#pragma unroll
                for (int q8 = 0; q8 < KT; q8++) {
                    pre[q8] = 0.f;
                    pu[q8] = make_float2(1.f, 0.f);
                    const int ti = c0 + q8;
                    if (ti >= n_terms) continue;  // uniform
                    const TermDev tm = sTerms[ti];
                    const int nf = term_nf(tm);
                    int rowoff[NFM];
                    float gq[NFM];
#pragma unroll
                    for (int q = 0; q < NFM; q++) {
                        const int f = q < nf ? term_flip(tm, q) : 0;
                        gq[q] = sbit(sp, f) ? 2.f : -2.f;  // -2 sigma_f
                        rowoff[q] = SYM ? f * S : f * ws;
                    }
                    float2 tp[E];
#pragma unroll
                    for (int j = 0; j < NG; j++) {
                        float2 acc[KB];
#pragma unroll
                        for (int i = 0; i < KB; i++) acc[i] = th[j * KB + i];
#pragma unroll
                        for (int q = 0; q < NFM; q++) {
                            if (q >= nf) break;  // uniform
                            const int row = SYM ? (int)sPerm[rowoff[q] + gs[j]] * ws : rowoff[q];
                            float2 w[KB];
                            Row<KB>::ld(W32 + row + gk[j], w);
                            const float2 G2 = make_float2(gq[q], gq[q]);
#pragma unroll
                            for (int i = 0; i < KB; i++) acc[i] = __ffma2_rn(G2, w[i], acc[i]);
                        }
#pragma unroll
                        for (int i = 0; i < KB; i++) tp[j * KB + i] = acc[i];
                    }
                    float re;
                    float2 u;
                    lnc_lane<E>(tp, nv, re, u);
                    pre[q8] = re - cre;
                    pu[q8] = cmulc(u, cu);
                }
                float R;
                float2 U;
                reduce_terms<KT>(pre, pu, lane, R, U);
                constexpr int sh = KT == 8 ? 2 : 3;
                const int ti = c0 + (lane >> sh);
                const bool owner = (lane & ((1 << sh) - 1)) == 0;
                if (owner && ti < n_terms) {
                    const TermDev tm = sTerms[ti];
                    const double2 val = vals[tm.voff + term_loc(tm, sp)];
                    if (val.x != 0.0 || val.y != 0.0) {
                        // visible bias of the flips (rbm_base.cpp:306-318)
                        const int nf = term_nf(tm);
                        double bx = 0.0, by = 0.0;
                        for (int q = 0; q < nf; q++) {
                            const int f = term_flip(tm, q);
                            const double sg = sbit(sp, f) ? -1.0 : 1.0;
                            const double2 v = sVb[vbi(f, n_vb, n)];
                            bx -= 2.0 * sg * v.x;
                            by -= 2.0 * sg * v.y;
                        }
                        const double lm = (double)R + bx;
                        double rx, ry;
                        if (fabs(lm) < 80.0) {
                            const float mag = exp_r((float)lm);
                            float sb, cb;
                            sincos_r((float)by, &sb, &cb);
                            rx = (double)(mag * (U.x * cb - U.y * sb));
                            ry = (double)(mag * (U.x * sb + U.y * cb));
                        } else {
                            const double mag = exp(lm);
                            double sb, cb;
                            sincos(by, &sb, &cb);
                            rx = mag * ((double)U.x * cb - (double)U.y * sb);
                            ry = mag * ((double)U.x * sb + (double)U.y * cb);
                        }
                        ex += val.x * rx - val.y * ry;
                        ey += val.x * ry + val.y * rx;
                    }
                }
            }
            ex = warp_sum(ex);
            ey = warp_sum(ey);
            if (lane == 0) a.eloc[b] = make_double2(ex, ey);
        }

        if (a.O) {
            __syncwarp();
            float2* Orow = reinterpret_cast<float2*>(a.O) + (size_t)b * m.P;
            if (SYM) {
                // v: sum_s sigma_{P_s(basis_q)}; h: sum_s tanh theta[k, s]
                for (int q = 0; q < n_vb; q++) {
                    float acc = 0.f;
                    for (int s = lane; s < S; s += 32) acc += sbit(sp, m.orbit[q * S + s]) ? -1.f : 1.f;
                    acc = warp_sum(acc);
                    if (lane == 0) Orow[q] = make_float2(acc, 0.f);
                }
                for (int k = 0; k < nh; k++) {
                    float2 acc = make_float2(0.f, 0.f);
                    for (int s = lane; s < S; s += 32) {
                        const float2 v = tn[k + nh * s];
                        acc.x += v.x;
                        acc.y += v.y;
                    }
                    acc.x = warp_sum(acc.x);
                    acc.y = warp_sum(acc.y);
                    if (lane == 0) Orow[n_vb + k] = acc;
                }
                // W[j, k]: sum_s sigma_{P_s^{-1}(j)} tanh theta[k, s]
                for (int j = lane; j < n; j += 32) {
                    for (int k0 = 0; k0 < nh; k0 += 4) {
                        float2 acc[4] = {};
                        for (int s = 0; s < S; s++) {
                            const float sg = sbit(sp, inv[s * n + j]) ? -1.f : 1.f;
                            const float2 G2 = make_float2(sg, sg);
#pragma unroll
                            for (int i = 0; i < 4; i++)
                                if (k0 + i < nh) acc[i] = __ffma2_rn(G2, tn[k0 + i + nh * s], acc[i]);
                        }
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            if (k0 + i < nh) Orow[n_vb + nh + j + n * (k0 + i)] = acc[i];
                    }
                }
            } else {
                for (int q = lane; q < n_vb; q += 32) Orow[q] = make_float2(sbit(sp, q) ? -1.f : 1.f, 0.f);
                for (int k = lane; k < nh; k += 32) Orow[n_vb + k] = tn[k];
                for (int k = 0; k < nh; k++) {
                    const float2 t = tn[k];
                    for (int j = lane; j < n; j += 32) {
                        const float sg = sbit(sp, j) ? -1.f : 1.f;
                        Orow[n_vb + nh + j + n * k] = make_float2(sg * t.x, sg * t.y);
                    }
                }
            }
        }
        __syncwarp();
    }
}

template <int KB, int NG, bool SYM, int NFM> const void* eloc_fn() {
    return reinterpret_cast<const void*>(eloc_kernel<KB, NG, SYM, NFM>);
}

template <int KB, int NG> const void* pick3(bool sym, int nfm) {
    if (sym) return nfm <= 2 ? eloc_fn<KB, NG, true, 2>() : eloc_fn<KB, NG, true, 6>();
    return nfm <= 2 ? eloc_fn<KB, NG, false, 2>() : eloc_fn<KB, NG, false, 6>();
}

// The instantiations are split over three files (one per group width KB) so
// that they compile in parallel: eloc_kb4.cu, eloc_kb2.cu, eloc_kb1.cu.
const void* pick_kb4(int ng, bool sym, int nfm);
const void* pick_kb2(int ng, bool sym, int nfm);
const void* pick_kb1(int ng, bool sym, int nfm);

}  // namespace eloc
}  // namespace rbmnqs
