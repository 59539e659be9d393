// eloc.cuh -- evaluation kernel of the FP32 hot path: local energy
// E_loc = sum_ops sum_l' H[l, l'] psi(sigma_l') / psi(sigma) (local_op.cpp:31-60)
// and log-derivatives O_k (rbm_base.cpp:194-217, rbm_symmetry.cpp:97-130) of
// every sampled configuration, one warp per configuration.
//
// Layout.  theta (T = nh S entries, t = k + nh s) is split into groups of KB
// consecutive hidden units k with the same symmetry index s; lane l owns
// groups g = l + 32 j (j < NG), so E = KB NG entries per lane, held as pairs
// of entries in structure-of-arrays form (real parts of two entries in one
// 64-bit register pair, imaginary parts in another) so that the ln cosh
// arithmetic runs on packed FP32x2 instructions.  Flipping site f adds
// -2 sigma_f W[P_s(f), k0 .. k0 + KB - 1] to a group: one byte of the
// symmetry table and one KB x 8-byte row segment of W, stored in shared
// memory in the same pair layout (re k0, re k0+1, im k0, im k0+1, ...), rows
// padded to an odd number of 16-byte units.  For symmetric machines the rows
// are stored in an order chosen on the host (wrank) so that the eight lanes
// of one 16-byte load phase, whose symmetry indices are consecutive, read
// rows in distinct bank groups.  Lanes whose groups lie beyond T read an
// all-zero row: their entries are 0 in theta and theta', and contribute the
// same exact constant to both ln cosh sums.
//
// E_loc.  The Hamiltonian comes as a table of terms (operator, flip mask,
// value per local configuration; TermDev).  For each term the lanes form
// theta' of their entries and the grouped ln cosh sum (one ex2, sin and cos
// per entry, one lg2 and rsqrt per four entries), giving a partial log
// magnitude and unit phase of psi'/psi.  KT terms at a time, the partials
// are reduced with a butterfly that leaves term q on lanes with
// (lane >> (5 - log2 KT)) == q, so the remaining per-term work (bias, exp and
// rotation, the matrix element, accumulation) runs once per term on
// different lanes.
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
// entries, 4-warp blocks at up to 72 registers (7 blocks, 28 warps per SM:
// 4096 samples, one per warp, in one wave of 148 SMs); above, 16-warp
// blocks at up to 128 registers.
__host__ __device__ constexpr int eloc_warps(int E) { return E <= 4 ? 4 : 16; }
__host__ __device__ constexpr int eloc_min_blocks(int E) { return E <= 4 ? 7 : 1; }

__host__ __device__ inline int a16(int x) { return (x + 15) & ~15; }

// Row stride of the W copy in shared memory, in floats: nh entries (plus KB
// zero entries for basic machines, read by groups beyond T) of 8 bytes,
// rounded up to an odd number of 16-byte units when rows are read 16 or 32
// bytes at a time.
__host__ __device__ inline int w32_stride(int nh, int kb, bool sym) {
    const int bytes = 8 * (nh + (sym ? 0 : kb));
    int u = (bytes + 15) / 16;
    if (kb > 1 && (u & 1) == 0) u++;
    return 4 * u;
}

// Row stride of the FP64 W copy in shared memory, in double2: an odd number
// of 16-byte units, so the eight lanes of a load phase reading rows of
// consecutive ranks hit distinct bank groups.
__host__ __device__ inline int w64_stride(int nh) { return (nh & 1) ? nh : nh + 1; }

// Shared-memory carve-up, the same arithmetic on host (sizing) and device.
struct ElocLayout {
    int w32, w64, perm, permw, inv, base, terms, diag, vals, vb, warp0, warp_bytes, total;
    int ws;    // row stride of the shared FP32 W copy (floats)
    int ws64;  // row stride of the shared FP64 W copy (double2)
    int w32_smem, w64_smem;
};

// Symmetric machines keep every table in shared memory (W in both
// precisions, the symmetry tables, the term values); basic machines read W
// from L2 when it does not fit (rows in their global layout).  Per warp:
// the configuration, tanh theta [T] and the spins as +-1 floats [n].
__host__ __device__ inline ElocLayout eloc_layout(const MachineDev& m, const TermTable& tt, int kb, int warps,
                                                  bool with_O, int budget) {
    ElocLayout L{};
    const bool sym = m.symmetric != 0;
    L.ws = w32_stride(m.nh, kb, sym);
    L.ws64 = w64_stride(m.nh);
    L.warp_bytes = a16(16 + m.T * 8 + m.n * 4);
    const int warps_b = warps * L.warp_bytes;
    const int base_b = a16(m.T * 16);
    const int perm_b = sym ? a16(m.n * (m.S + 1)) : 0;
    const int permw_b = sym ? a16(2 * m.n * (m.S + 1)) : 0;
    const int terms_b = a16((tt.n_terms + tt.n_diag) * (int)sizeof(TermDev));
    const int vb_b = a16(m.n_vb * 16);
    const int w32_b = a16((m.n + 1) * L.ws * 4), vals_b = a16(tt.n_vals * 16);
    const int w64_b = a16(m.n * L.ws64 * 16);
    const int inv_b = (sym && with_O) ? a16(m.n * m.S) : 0;
    int need = warps_b + base_b + perm_b + permw_b + terms_b + vb_b + vals_b + inv_b;
    if (sym) need += w32_b + w64_b;
    L.w32_smem = sym || need + w32_b <= budget;
    if (!sym && L.w32_smem) need += w32_b;
    L.w64_smem = sym || need + w64_b <= budget;
    int off = 0;
    L.w32 = off;
    off += L.w32_smem ? w32_b : 0;
    L.w64 = off;
    off += L.w64_smem ? w64_b : 0;
    L.perm = off;
    off += perm_b;
    L.permw = off;
    off += permw_b;
    L.inv = off;
    off += inv_b;
    L.base = off;
    off += base_b;
    L.terms = off;
    L.diag = off + tt.n_terms * (int)sizeof(TermDev);
    off += terms_b;
    L.vals = off;
    off += vals_b;
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
__device__ __forceinline__ int term_flip(const TermDev& t, int q) {
    return q < 4 ? byte_of(t.flip0, q) : byte_of(t.flip1, q - 4);
}
__device__ __forceinline__ int term_site(const TermDev& t, int q) {
    return q < 4 ? byte_of(t.site0, q) : byte_of(t.site1, q - 4);
}
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

__device__ __forceinline__ float4 lds128(uint32_t a) {
    float4 v;
    asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ float2 lds64(uint32_t a) {
    float2 v;
    asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ uint32_t lds16(uint32_t a) {
    uint32_t v;
    asm("ld.shared.u16 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ uint32_t lds8(uint32_t a) {
    uint32_t v;
    asm("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}

// ln cosh over E entries held as structure-of-arrays pairs (ar[p] = real
// parts of entries 2p, 2p+1; ai[p] = imaginary parts), by the formula of
// common.cuh (lnc_lane): with z = exp(-2|a|), cosh(a + ib) is proportional to
// (1 + z) cos b + i (1 - z) sin(sgn(a) b).  re = sum |a| + ln|prod| and u =
// its unit phase, ln 2 per entry left out; the factors are multiplied in
// groups of four (two pairs), one lg2 and one rsqrt per group.
template <int E>
__device__ __forceinline__ void lnc_pairs(const float2 (&ar)[E / 2], const float2 (&ai)[E / 2], float& re,
                                          float2& u) {
    constexpr int NP = E / 2;
    float2 as2 = make_float2(0.f, 0.f);
    float l2 = 0.f;
    float2 P = make_float2(1.f, 0.f);
#pragma unroll
    for (int g = 0; g < NP; g += 2) {
        float2 Gx = make_float2(1.f, 1.f), Gy = make_float2(0.f, 0.f);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            if (g + h >= NP) break;
            const float2 A = ar[g + h], B = ai[g + h];
            const uint32_t ax = __float_as_uint(A.x), ay = __float_as_uint(A.y);
            const float2 aa = make_float2(__uint_as_float(ax & 0x7fffffffu), __uint_as_float(ay & 0x7fffffffu));
            const float2 bs = make_float2(__uint_as_float(__float_as_uint(B.x) ^ (ax & 0x80000000u)),
                                          __uint_as_float(__float_as_uint(B.y) ^ (ay & 0x80000000u)));
            as2 = __fadd2_rn(as2, aa);
            const float2 t = __fmul2_rn(aa, make_float2(-2.88539008177792681f, -2.88539008177792681f));
            const float2 z = make_float2(ftz_ex2(t.x), ftz_ex2(t.y));
            // b reduced to [-pi, pi] (Cody-Waite, as reduce_2pi); k = rint(b / 2 pi)
            // by adding and subtracting 1.5 2^23 (exact for |b / 2 pi| < 2^22)
            float2 k = __ffma2_rn(bs, make_float2(0.159154943091895336f, 0.159154943091895336f),
                                  make_float2(12582912.f, 12582912.f));
            k = __fadd2_rn(k, make_float2(-12582912.f, -12582912.f));
            float2 r = __ffma2_rn(k, make_float2(-6.28318548202514648f, -6.28318548202514648f), bs);
            r = __ffma2_rn(k, make_float2(1.74845553146951e-07f, 1.74845553146951e-07f), r);
            const float2 s = make_float2(ftz_sin(r.x), ftz_sin(r.y));
            const float2 c = make_float2(ftz_cos(r.x), ftz_cos(r.y));
            const float2 X = __ffma2_rn(z, c, c);
            const float2 Y = __ffma2_rn(make_float2(-z.x, -z.y), s, s);
            const float2 nx = __ffma2_rn(Gx, X, __fmul2_rn(Gy, make_float2(-Y.x, -Y.y)));
            const float2 ny = __ffma2_rn(Gx, Y, __fmul2_rn(Gy, X));
            Gx = nx;
            Gy = ny;
        }
        const float2 G = make_float2(Gx.x * Gx.y - Gy.x * Gy.y, Gx.x * Gy.y + Gy.x * Gx.y);
        const float m2 = G.x * G.x + G.y * G.y;
        const bool ok = m2 >= 1.17549435e-38f;
        l2 += ok ? ftz_lg2(m2) : __int_as_float(0xff800000u);  // a zero of cosh: -inf
        const float inv = ok ? ftz_rsqrt(m2) : 0.f;
        P = cmul(P, make_float2(G.x * inv, G.y * inv));
    }
    re = as2.x + as2.y + 0.346573590279972655f * l2;  // (ln 2 / 2) lg2
    u = P;
}

// Butterfly reduce-scatter of KT per-lane partials (log magnitude summed,
// unit phase multiplied): afterwards every lane holds the total of term
// (lane >> (5 - log2 KT)), the same on the 32 / KT lanes of that term.
template <int KT>
__device__ __forceinline__ void reduce_terms(float (&re)[KT], float2 (&u)[KT], int lane, float& R, float2& U) {
    static_assert(KT == 4 || KT == 8, "4 or 8 terms per round");
#pragma unroll
    for (int stage = 0; stage < (KT == 8 ? 3 : 2); stage++) {
        const int off = 16 >> stage;
        const int half = (KT >> stage) >> 1;
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

// W row segment of group j as structure-of-arrays pairs, from the shared
// copy (pair layout, byte address) or, for basic machines whose W does not
// fit, from the global copy (site-major, complex interleaved).
template <int KB>
__device__ __forceinline__ void seg_smem(uint32_t a, float2 (&r)[KB / 2 > 0 ? KB / 2 : 1],
                                         float2 (&i)[KB / 2 > 0 ? KB / 2 : 1]) {
    if constexpr (KB == 4) {
        const float4 v0 = lds128(a), v1 = lds128(a + 16);
        r[0] = make_float2(v0.x, v0.y);
        i[0] = make_float2(v0.z, v0.w);
        r[1] = make_float2(v1.x, v1.y);
        i[1] = make_float2(v1.z, v1.w);
    } else if constexpr (KB == 2) {
        const float4 v0 = lds128(a);
        r[0] = make_float2(v0.x, v0.y);
        i[0] = make_float2(v0.z, v0.w);
    }
}
template <int KB>
__device__ __forceinline__ void seg_global(const float2* p, float2 (&r)[KB / 2 > 0 ? KB / 2 : 1],
                                           float2 (&i)[KB / 2 > 0 ? KB / 2 : 1]) {
    if constexpr (KB >= 2) {
#pragma unroll
        for (int q = 0; q < KB / 2; q++) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(p) + q);
            r[q] = make_float2(v.x, v.z);
            i[q] = make_float2(v.y, v.w);
        }
    }
}

template <int KB, int NG, bool SYM, int NFM>
__global__ void __launch_bounds__(32 * eloc_warps(KB* NG), eloc_min_blocks(KB* NG))
    eloc_kernel(const EvalArgs a, const ElocLayout L) {
    constexpr int E = KB * NG;
    constexpr int NP = E / 2;               // entry pairs per lane
    constexpr int WARPS = eloc_warps(E);
    constexpr int KT = E >= 16 ? 4 : 8;     // terms per reduction round
    static_assert(E % 2 == 0, "entries per lane come in pairs");
    extern __shared__ __align__(16) unsigned char smem[];
    const MachineDev& m = a.m;
    const int n = m.n, nh = m.nh, S = m.S, T = m.T, n_vb = m.n_vb;
    const int SP = S + 1;  // symmetry-table row: S entries and the zero-row column
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int n_terms = a.tt.n_terms, n_diag = a.tt.n_diag;
    const int ws = L.ws;

    // ---- block tables
    float* sW32 = reinterpret_cast<float*>(smem + L.w32);
    double2* sW64 = reinterpret_cast<double2*>(smem + L.w64);
    uint8_t* sPerm = smem + L.perm;
    uint16_t* sPermW = reinterpret_cast<uint16_t*>(smem + L.permw);
    uint8_t* sInv = smem + L.inv;
    double2* sBase = reinterpret_cast<double2*>(smem + L.base);
    TermDev* sTerms = reinterpret_cast<TermDev*>(smem + L.terms);
    TermDev* sDiag = reinterpret_cast<TermDev*>(smem + L.diag);
    double2* sVals = reinterpret_cast<double2*>(smem + L.vals);
    double2* sVb = reinterpret_cast<double2*>(smem + L.vb);
    auto rk = [&](int r) { return (SYM && a.wrank) ? (int)a.wrank[r] : r; };
    if (L.w32_smem) {
        // pair layout: entry k of row r at (k - k%KB) * 2 + {re, im} offsets
        const int rows = n + 1, per = ws;
        for (int i = tid; i < rows * per; i += nthr) sW32[i] = 0.f;
        __syncthreads();
        for (int i = tid; i < n * nh; i += nthr) {
            const int r = i / nh, k = i % nh, kk = k % KB, k0 = k - kk;
            const float2 w = m.W32[i];
            float* row = sW32 + rk(r) * per + 2 * k0;
            const int re_off = KB == 1 ? 0 : 4 * (kk >> 1) + (kk & 1);
            const int im_off = KB == 1 ? 1 : re_off + 2;
            row[re_off] = w.x;
            row[im_off] = w.y;
        }
    }
    const int ws64 = L.w64_smem ? L.ws64 : nh;
    if (L.w64_smem)
        for (int i = tid; i < n * nh; i += nthr) sW64[rk(i / nh) * ws64 + i % nh] = m.W64[i];
    if (SYM) {
        // symmetry table: W row rank (FP64 copy) and FP32-copy byte offset;
        // column S is the zero row n
        for (int i = tid; i < n * SP; i += nthr) {
            const int f = i / SP, s = i % SP;
            const int r = s < S ? rk(m.perm[f * S + s]) : n;
            sPerm[i] = (uint8_t)r;
            sPermW[i] = (uint16_t)(4 * r * ws);
        }
        if (a.O)
            for (int i = tid; i < n * S; i += nthr) sInv[i] = m.inv[i];
    }
    for (int i = tid; i < n_terms; i += nthr) sTerms[i] = a.tt.terms[i];
    for (int i = tid; i < n_diag; i += nthr) sDiag[i] = a.tt.diag[i];
    for (int i = tid; i < a.tt.n_vals; i += nthr) sVals[i] = a.tt.vals[i];
    for (int i = tid; i < n_vb; i += nthr) sVb[i] = m.vb[i];
    __syncthreads();
    const double2* W64 = (SYM || L.w64_smem) ? sW64 : m.W64;
    // theta of the all-up configuration (FP64): hb_k + sum_f W[P_s(f), k]
    for (int t = tid; t < T; t += nthr) {
        const int k = t % nh, s = t / nh;
        double2 acc = m.hb[k];
        for (int f = 0; f < n; f++) {
            const double2 w = W64[(SYM ? (int)sPerm[f * SP + s] : f) * ws64 + k];
            acc.x += w.x;
            acc.y += w.y;
        }
        sBase[t] = acc;
    }
    __syncthreads();

    const int warp = tid >> 5, lane = tid & 31;
    unsigned char* wbase = smem + L.warp0 + warp * L.warp_bytes;
    float2* tn = reinterpret_cast<float2*>(wbase + 16);
    float* sgn = reinterpret_cast<float*>(wbase + 16 + T * 8);  // sigma_i as +-1
    const uint32_t wsa = (uint32_t)__cvta_generic_to_shared(sW32);
    const uint32_t pwa = (uint32_t)__cvta_generic_to_shared(sPermW);
    // the lane's groups: symmetry index s, first hidden unit k0, validity.
    // Groups beyond T read the zero row: symmetry column S (symmetric) or
    // the row's zero tail at k0 = nh (basic, shared copy).
    const int G = T / KB, NGK = nh / KB;
    // per group: byte address of the group's entry in the symmetry row of
    // site 0 (add 2 SP f for site f) and byte address of its first entry in
    // a W row (add the row's offset); s and k0 are recovered from them
    uint32_t pw0[NG], go8[NG];
    uint32_t vmask = 0;
#pragma unroll
    for (int j = 0; j < NG; j++) {
        const int g = lane + 32 * j;
        const bool ok = g < G;
        const int s = ok ? g / NGK : S;
        const int k0 = ok ? (g % NGK) * KB : (SYM ? 0 : nh);
        pw0[j] = pwa + 2u * (uint32_t)s;
        go8[j] = wsa + 8u * (uint32_t)k0;
        vmask |= ok ? 1u << j : 0u;
    }
    auto g_s = [&](int j) { return (int)((pw0[j] - pwa) >> 1); };
    auto g_k = [&](int j) { return (int)((go8[j] - wsa) >> 3); };

    for (int b = blockIdx.x * WARPS + warp; b < a.B; b += gridDim.x * WARPS) {
        uint32_t sp[4];
#pragma unroll
        for (int w = 0; w < 4; w++) sp[w] = a.spins[4 * b + w];
        if (a.O)
            for (int i = lane; i < n; i += 32) sgn[i] = sbit(sp, i) ? -1.f : 1.f;

        // ---- theta in FP64 (down spins subtracted from the all-up table),
        // rounded to FP32 pairs; tanh theta in FP64 into the warp's scratch
        float2 thr[NP], thi[NP];
#pragma unroll
        for (int j = 0; j < NG; j++) {
            double2 acc[KB];
            const bool ok = (vmask >> j) & 1u;
            const int gsj = g_s(j), gkj = g_k(j);
            const int t0 = gkj + nh * gsj;
#pragma unroll
            for (int i = 0; i < KB; i++) acc[i] = ok ? sBase[t0 + i] : make_double2(0, 0);
            if (ok) {
#pragma unroll
                for (int wd = 0; wd < 4; wd++) {
                    uint32_t bits = sp[wd];
                    while (bits) {
                        const int f = 32 * wd + __ffs(bits) - 1;
                        bits &= bits - 1;
                        const int row = SYM ? (int)sPerm[f * SP + gsj] : f;
                        const double2* wr = W64 + row * ws64 + gkj;
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
                const int e = j * KB + i;
                if (e & 1) {
                    thr[e >> 1].y = (float)acc[i].x;
                    thi[e >> 1].y = (float)acc[i].y;
                } else {
                    thr[e >> 1].x = (float)acc[i].x;
                    thi[e >> 1].x = (float)acc[i].y;
                }
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
                const double2 v = sVals[td.voff + term_loc(td, sp)];
                ex += v.x;
                ey += v.y;
            }
            float cre;
            float2 cu;
            lnc_pairs<E>(thr, thi, cre, cu);
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
                    // theta' = theta - 2 sigma_f W[..] over the flips; an
                    // off-diagonal term flips at least one site, so the
                    // first flip reads theta and writes theta' directly
                    // (no per-term copy of the lane's theta registers)
                    float2 tr[NP], tq[NP];
#pragma unroll
                    for (int q = 0; q < NFM; q++) {
                        if (q > 0 && q >= nf) break;  // uniform
                        const int f = term_flip(tm, q);
                        const float g = sbit(sp, f) ? 2.f : -2.f;  // -2 sigma_f
                        const float2 g2 = make_float2(g, g);
                        if constexpr (KB >= 2) {
#pragma unroll
                            for (int j = 0; j < NG; j++) {
                                float2 ur[KB / 2], ui[KB / 2];
                                if (SYM) {
                                    const uint32_t ro = lds16(pw0[j] + 2u * (uint32_t)(f * SP));
                                    seg_smem<KB>(go8[j] + ro, ur, ui);
                                } else if (L.w32_smem) {
                                    seg_smem<KB>(go8[j] + 4u * (uint32_t)(f * ws), ur, ui);
                                } else {
                                    const bool ok = (vmask >> j) & 1u;
                                    seg_global<KB>(m.W32 + (ok ? f : n) * nh + (ok ? g_k(j) : 0), ur, ui);
                                }
#pragma unroll
                                for (int h = 0; h < KB / 2; h++) {
                                    const int pi = j * (KB / 2) + h;
                                    tr[pi] = __ffma2_rn(g2, ur[h], q == 0 ? thr[pi] : tr[pi]);
                                    tq[pi] = __ffma2_rn(g2, ui[h], q == 0 ? thi[pi] : tq[pi]);
                                }
                            }
                        } else {
                            // one entry per group: a pair spans groups 2p, 2p + 1
#pragma unroll
                            for (int p = 0; p < NP; p++) {
                                float2 w[2];
#pragma unroll
                                for (int h = 0; h < 2; h++) {
                                    const int j = 2 * p + h;
                                    if (SYM) {
                                        const uint32_t ro = lds16(pw0[j] + 2u * (uint32_t)(f * SP));
                                        w[h] = lds64(go8[j] + ro);
                                    } else if (L.w32_smem) {
                                        w[h] = lds64(go8[j] + 4u * (uint32_t)(f * ws));
                                    } else {
                                        const bool ok = (vmask >> j) & 1u;
                                        w[h] = __ldg(m.W32 + (ok ? f : n) * nh + (ok ? g_k(j) : 0));
                                    }
                                }
                                tr[p] = __ffma2_rn(g2, make_float2(w[0].x, w[1].x), q == 0 ? thr[p] : tr[p]);
                                tq[p] = __ffma2_rn(g2, make_float2(w[0].y, w[1].y), q == 0 ? thi[p] : tq[p]);
                            }
                        }
                    }
                    float re;
                    float2 u;
                    lnc_pairs<E>(tr, tq, re, u);
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
                    const double2 val = sVals[tm.voff + term_loc(tm, sp)];
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
                // W[j, k]: sum_s sigma_{P_s^{-1}(j)} tanh theta[k, s].  With
                // n a multiple of 128 and nh of 4, each lane takes four
                // consecutive sites: one 32-bit load gives their four
                // inverse-symmetry bytes, two 16-byte loads the four tanh
                // values they share (same sums, same order per output)
                if (n % 128 == 0 && nh % 4 == 0) {
                    for (int jb = 4 * lane; jb < n; jb += 128) {
                        for (int k0 = 0; k0 < nh; k0 += 4) {
                            float2 acc[4][4] = {};
                            for (int s = 0; s < S; s++) {
                                const uint32_t iv = *reinterpret_cast<const uint32_t*>(sInv + s * n + jb);
                                const float4 t01 = *reinterpret_cast<const float4*>(tn + k0 + nh * s);
                                const float4 t23 = *reinterpret_cast<const float4*>(tn + k0 + 2 + nh * s);
                                const float2 t[4] = {make_float2(t01.x, t01.y), make_float2(t01.z, t01.w),
                                                     make_float2(t23.x, t23.y), make_float2(t23.z, t23.w)};
#pragma unroll
                                for (int jj = 0; jj < 4; jj++) {
                                    const float sg = sgn[(iv >> (8 * jj)) & 0xffu];
                                    const float2 G2 = make_float2(sg, sg);
#pragma unroll
                                    for (int i = 0; i < 4; i++) acc[jj][i] = __ffma2_rn(G2, t[i], acc[jj][i]);
                                }
                            }
#pragma unroll
                            for (int i = 0; i < 4; i++)
#pragma unroll
                                for (int jj = 0; jj < 4; jj++)
                                    Orow[n_vb + nh + jb + jj + n * (k0 + i)] = acc[jj][i];
                        }
                    }
                } else
                for (int j = lane; j < n; j += 32) {
                    for (int k0 = 0; k0 < nh; k0 += 4) {
                        float2 acc[4] = {};
                        for (int s = 0; s < S; s++) {
                            const float sg = sgn[sInv[s * n + j]];
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
                        const float sg = sgn[j];
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
