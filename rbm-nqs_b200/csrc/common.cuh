// common.cuh -- device helpers shared by the sm_100a kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rbmnqs {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------- complex --
template <typename R> struct c2t;
template <> struct c2t<float> { using type = float2; };
template <> struct c2t<double> { using type = double2; };
template <typename R> using C2 = typename c2t<R>::type;

template <typename R> __device__ __forceinline__ C2<R> mk(R x, R y) { return {x, y}; }
template <typename T> __device__ __forceinline__ T cmul(T a, T b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T> __device__ __forceinline__ T cmulc(T a, T b) {  // a * conj(b)
    return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}

// ------------------------------------------------------------- Philox ---
// Philox4x32-10 (Salmon et al., SC'11).  Counter layout shared with the
// oracle: {proposal index, epoch, chain, stream}, key = 64-bit seed.
__device__ __forceinline__ uint4 philox4x32(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// 24-bit uniform in [0, 1): exactly representable in float and double.
template <typename R> __device__ __forceinline__ R unit24(uint32_t x) {
    return (R)(x >> 8) * (R)(1.0 / 16777216.0);
}
__device__ __forceinline__ uint32_t pick(uint32_t x, uint32_t n) { return __umulhi(x, n); }

// ------------------------------------------------------ warp reductions --
template <typename R> __device__ __forceinline__ R warp_sum(R v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
template <typename T> __device__ __forceinline__ T warp_cprod(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T w;
        w.x = __shfl_xor_sync(kFull, v.x, o);
        w.y = __shfl_xor_sync(kFull, v.y, o);
        v = cmul(v, w);
    }
    return v;
}

// -------------------------------------------------------- ln cosh math --
// For x = a + ib with z = exp(-2|a|):
//   cosh x = e^{|a|}/2 * (X + i sgn(a) Y),  X = (1+z) cos b,  Y = (1-z) sin b
// so ln cosh x = |a| - ln 2 + ln|X + i sgn(a) Y| + i arg(X + i sgn(a) Y).
// This is the reference's overflow-free form (math.cpp:37-56) rearranged so
// that one exp, one sincos and one log serve the real part.  The constant
// -ln 2 is left out (it cancels in every psi ratio) and added back by log psi.
//
// FP32 path: Cody-Waite reduction of b to [-pi, pi] keeps the hardware
// sin/cos approximations at their small-argument accuracy.
__device__ __forceinline__ float reduce_2pi(float b) {
    const float k = rintf(b * 0.159154943091895336f);
    float r = fmaf(-k, 6.28318548202514648f, b);
    return fmaf(-k, -1.74845553146951e-07f, r);
}

// The FP32 forms issue the hardware approximations in their flush-to-zero
// variants (the non-flushing ones add a denormal test and rescale around
// each): a denormal z = e^{-2|a|} (|a| > 43) becomes 0, the exact limit; a
// denormal argument of the log (a zero of cosh to FP32 precision) gives
// -inf, a state of vanishing amplitude.
__device__ __forceinline__ float ftz_ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ftz_lg2(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ftz_sin(float x) {
    float y;
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ftz_cos(float x) {
    float y;
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ftz_rsqrt(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ void sincos_r(float b, float* s, float* c) {
    const float r = reduce_2pi(b);
    *s = ftz_sin(r);
    *c = ftz_cos(r);
}
__device__ __forceinline__ void sincos_r(double b, double* s, double* c) { sincos(b, s, c); }
__device__ __forceinline__ float exp_r(float x) { return ftz_ex2(x * 1.44269504088896341f); }
__device__ __forceinline__ double exp_r(double x) { return exp(x); }
__device__ __forceinline__ float log_r(float x) { return ftz_lg2(x) * 0.693147180559945309f; }
__device__ __forceinline__ double log_r(double x) { return log(x); }
__device__ __forceinline__ float rsqrt_r(float x) { return ftz_rsqrt(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }

// Real part only (Metropolis acceptance needs |psi'/psi|).
template <typename R> __device__ __forceinline__ R lnc_re(R a, R b) {
    const R aa = fabs(a);
    const R z = exp_r((R)-2 * aa);
    R s, c;
    sincos_r(b, &s, &c);
    const R X = ((R)1 + z) * c, Y = ((R)1 - z) * s;
    return aa + (R)0.5 * log_r(X * X + Y * Y);
}

// Real part and unit phase.
template <typename R> __device__ __forceinline__ void lnc_full(R a, R b, R& re, R& ux, R& uy) {
    const R aa = fabs(a);
    const R z = exp_r((R)-2 * aa);
    R s, c;
    sincos_r(b, &s, &c);
    const R X = ((R)1 + z) * c;
    const R Y = copysign((R)1 - z, a) * s;
    const R m2 = X * X + Y * Y;
    re = aa + (R)0.5 * log_r(m2);
    const R inv = m2 > (R)0 ? rsqrt_r(m2) : (R)0;
    ux = X * inv;
    uy = Y * inv;
}

// FP32 sum of ln cosh over a lane's valid entries x[e] (e < nv): re = sum |a|
// + ln|prod (X + i sgn(a) Y)| and u = the unit phase of that product (ln 2
// per entry left out, as in lnc_full).  The factors are multiplied in groups
// of four (|X + iY| <= 2, so a group's product stays in the FP32 range), with
// one lg2 and one rsqrt per group instead of one per entry.  A group whose
// |product|^2 is below the smallest normal float counts as a zero of cosh:
// re = -inf, u = 0.
template <int E> __device__ __forceinline__ void lnc_lane(const float2 (&x)[E], int nv, float& re, float2& u) {
    float asum = 0.f, l2 = 0.f;
    float2 P = make_float2(1.f, 0.f);
#pragma unroll
    for (int g = 0; g < E; g += 4) {
        if (g >= nv) break;
        float2 G = make_float2(1.f, 0.f);
#pragma unroll
        for (int j = 0; j < 4 && g + j < E; j++) {
            if (g + j >= nv) break;
            const float a = x[g + j].x, aa = fabsf(a);
            const float z = exp_r(-2.f * aa);
            float s, c;
            sincos_r(x[g + j].y, &s, &c);
            const float2 f = make_float2((1.f + z) * c, copysignf(1.f - z, a) * s);
            asum += aa;
            G = cmul(G, f);
        }
        const float m2 = G.x * G.x + G.y * G.y;
        const bool ok = m2 >= 1.17549435e-38f;
        l2 += ok ? ftz_lg2(m2) : __int_as_float(0xff800000u);  // -inf
        const float inv = ok ? ftz_rsqrt(m2) : 0.f;
        P = cmul(P, make_float2(G.x * inv, G.y * inv));
    }
    re = asum + 0.346573590279972655f * l2;  // (ln 2 / 2) lg2
    u = P;
}

// tanh(a + ib) = [sgn(a)(1 - z^2) + i 4z sin b cos b] / (X^2 + Y^2), the
// denominator 1 + z^2 + 2z cos 2b written as the sum of squares
// X^2 + Y^2 = ((1+z) cos b)^2 + ((1-z) sin b)^2, which does not cancel near
// the poles of tanh; 1 - z comes from expm1 so small |a| keeps its digits.
__device__ __forceinline__ float expm1_r(float x) { return expm1f(x); }
__device__ __forceinline__ double expm1_r(double x) { return expm1(x); }

template <typename R> __device__ __forceinline__ C2<R> ctanh_r(R a, R b) {
    const R aa = fabs(a);
    const R omz = -expm1_r((R)-2 * aa);  // 1 - z
    const R z = (R)1 - omz;
    R s, c;
    sincos_r(b, &s, &c);
    const R X = ((R)1 + z) * c, Y = omz * s;
    const R inv = (R)1 / (X * X + Y * Y);
    return mk<R>(copysign(omz * ((R)1 + z), a) * inv, (R)4 * z * s * c * inv);
}

// Raise (never lower) a kernel's dynamic shared-memory limit.  The limit is a
// per-function attribute shared by every session in the process, and launches
// already captured into CUDA graphs keep the size they were recorded with, so
// it only ever grows to the largest size any session needs.
cudaError_t ensure_dynamic_smem(const void* fn, int bytes);

}  // namespace rbmnqs
