// Device-side building blocks shared by the lattice kernels: the counter-based
// hash noise, the V' sources and the three state storages.
//
// Reference citations: R = simulation/latticeSimeRescale_numba.py,
//                      C = simulation/latticeSimComplex_numba.py.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "tipt.h"

namespace tipt {

constexpr uint64_t kPass2Mul = 73856093ull;   // R:2518 (pass 2 / midpoint)
constexpr uint64_t kPass4Mul = 19349669ull;   // R:2643 (pass 4)
constexpr uint64_t kSeedStride = 0x9E3779B97F4A7C15ull;
constexpr double kTwoPiLit = 6.283185307179586;  // literal of R:2520

// ---------------------------------------------------------------- noise ----
// R:2322-2336 _hash_rng_pair: splitmix-style mix -> two 53-bit uniforms.  The
// second mix of the reference kernel is partial (no >>27 round); u1 >= 1e-12.
__device__ __forceinline__ void hash_pair(uint64_t x, double& u1, double& u2) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x = x ^ (x >> 31);
    u1 = (double)(x >> 11) * (1.0 / 9007199254740992.0);
    x = (x * 0x2545F4914F6CDD1Dull) ^ 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = x ^ (x >> 31);
    u2 = (double)(x >> 11) * (1.0 / 9007199254740992.0);
    u1 = u1 < 1e-12 ? 1e-12 : u1;
}

// R:2515-2518: key = uint64(site*mul) ^ uint64(step); the seed term is an
// extension that leaves the reference key unchanged at seed = 0.
__device__ __forceinline__ uint64_t noise_key(uint64_t site, uint64_t step, uint64_t mul,
                                              uint64_t seed) {
    return ((site * mul) ^ step) + seed * kSeedStride;
}

// R:2519-2521 Box-Muller radius and angle, FP64 (the reference's precision).
__device__ __forceinline__ double bm_radius(double u1) { return sqrt(-2.0 * log(u1)); }
__device__ __forceinline__ double gauss_cos(uint64_t key) {
    double u1, u2;
    hash_pair(key, u1, u2);
    return bm_radius(u1) * cos(kTwoPiLit * u2);
}
// C:2965-2970: the complex field draws one pair per site: cos -> pi1, sin -> pi2.
__device__ __forceinline__ void gauss_pair(uint64_t key, double& z1, double& z2) {
    double u1, u2;
    hash_pair(key, u1, u2);
    double r = bm_radius(u1);
    double s, c;
    sincos(kTwoPiLit * u2, &s, &c);
    z1 = r * c;
    z2 = r * s;
}

// FP32 Box-Muller for the compensated-FP32 storage.  The hash is the same
// integer computation; only the Gaussian transform runs in FP32, from the exact
// 53-bit integers m1, m2 (u = m * 2^-53), with argument reductions done exactly
// in integer arithmetic and short series on the reduced ranges:
//  * log(u1): u1 = 2^(e-53) (1 + g) with 1 + g in [3/4, 3/2) and g formed by an
//    exact integer subtraction; log(1 + g) = 2 atanh(s), s = g / (2 + g),
//    |s| <= 1/5, summed as 2 s (1 + s^2/3 + s^4/5 + ... + s^10/11) (the atanh
//    series; truncation < 4e-10 relative).  The reference's clamp
//    u1 >= 1e-12 is m1 <= 9007.
//  * cos/sin(2 pi u2): 2 u2 = m2 * 2^-52; the nearest quarter turn is taken from
//    the integer (exact), the remainder x lies in [-pi/4, pi/4] and the Taylor
//    series of sin (to x^9) and cos (to x^10) are truncated below 3e-9.
//  * sqrt via rsqrt and one Newton step.
// z agrees with the FP64 reference value to a few FP32 ulps.
__device__ __forceinline__ void hash_bits(uint64_t x, uint64_t& m1, uint64_t& m2) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x = x ^ (x >> 31);
    m1 = x >> 11;
    x = (x * 0x2545F4914F6CDD1Dull) ^ 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = x ^ (x >> 31);
    m2 = x >> 11;
}

constexpr float kLn2Hi = 0.693147182464599609375f;   // ln 2 rounded to FP32
constexpr float kLn2Lo = -1.904654299957768e-09f;    // ln 2 - kLn2Hi
constexpr float kLog1em12 = -27.631021115928547f;    // log(1e-12)

__device__ __forceinline__ float log_u1_f(uint64_t m1) {
    if (m1 <= 9007ull) return kLog1em12;
    const int e = 63 - __clzll((long long)m1);            // m1 in [2^e, 2^(e+1))
    const int ep = ((m1 >> (e - 1)) & 1ull) ? e + 1 : e;   // m1 / 2^ep in [3/4, 3/2)
    const long long gi = (long long)m1 - (1ll << ep);      // exact
    const float g = __fmul_rn(__ll2float_rn(gi), __int_as_float((127 - ep) << 23));
    const float s = __fdividef(g, __fadd_rn(2.0f, g));
    const float w = __fmul_rn(s, s);
    float poly = __fmaf_rn(w, 1.0f / 11.0f, 1.0f / 9.0f);
    poly = __fmaf_rn(w, poly, 1.0f / 7.0f);
    poly = __fmaf_rn(w, poly, 1.0f / 5.0f);
    poly = __fmaf_rn(w, poly, 1.0f / 3.0f);
    poly = __fmul_rn(w, poly);                             // s^2/3 + ... + s^10/11
    const float two_s = __fadd_rn(s, s);
    const float l1p = __fmaf_rn(two_s, poly, two_s);       // 2 s (1 + poly)
    const float k = (float)(ep - 53);
    return __fmaf_rn(k, kLn2Hi, __fmaf_rn(k, kLn2Lo, l1p));
}

__device__ __forceinline__ void cossin_2pi_f(uint64_t m2, float& c, float& s) {
    // 2 u2 = m2 * 2^-52 = q/2 + r * 2^-52: q quarter turns (the multiple of
    // 2^51 nearest m2) plus a remainder |r| <= 2^50, i.e. |x| <= pi/4
    const uint32_t q = (uint32_t)((m2 + (1ull << 50)) >> 51);        // 0..4
    const long long r = (long long)m2 - ((long long)q << 51);
    const float x = __fmul_rn(__ll2float_rn(r), 6.97573699e-16f);    // pi * 2^-52
    const float x2 = __fmul_rn(x, x);
    float sp = __fmaf_rn(x2, 2.75573192e-6f, -1.98412698e-4f);       // 1/9!, -1/7!
    sp = __fmaf_rn(x2, sp, 8.33333333e-3f);                          // 1/5!
    sp = __fmaf_rn(x2, sp, -1.66666667e-1f);                         // -1/3!
    const float sn = __fmaf_rn(__fmul_rn(x2, x), sp, x);
    float cp = __fmaf_rn(x2, -2.75573192e-7f, 2.48015873e-5f);       // -1/10!, 1/8!
    cp = __fmaf_rn(x2, cp, -1.38888889e-3f);                         // -1/6!
    cp = __fmaf_rn(x2, cp, 4.16666667e-2f);                          // 1/4!
    cp = __fmaf_rn(x2, cp, -0.5f);
    const float cs = __fmaf_rn(x2, cp, 1.0f);
    // rotate by q quarter turns
    const uint32_t qq = q & 3u;
    const float a = (qq & 1u) ? sn : cs;
    const float b = (qq & 1u) ? cs : sn;
    c = (qq == 1u || qq == 2u) ? -a : a;
    s = (qq >= 2u) ? -b : b;
}

__device__ __forceinline__ float bm_radius_f(uint64_t m1) {
    const float v = __fmul_rn(-2.0f, log_u1_f(m1));   // > 0
    const float y = rsqrtf(v);
    const float r = __fmul_rn(v, y);
    return __fmaf_rn(__fmul_rn(0.5f, y), __fmaf_rn(-r, r, v), r);  // one Newton step
}

__device__ __forceinline__ float gauss_cos_f(uint64_t key) {
    uint64_t m1, m2;
    hash_bits(key, m1, m2);
    float c, s;
    cossin_2pi_f(m2, c, s);
    return __fmul_rn(bm_radius_f(m1), c);
}

__device__ __forceinline__ void gauss_pair_f(uint64_t key, float& z1, float& z2) {
    uint64_t m1, m2;
    hash_bits(key, m1, m2);
    float c, s;
    cossin_2pi_f(m2, c, s);
    const float r = bm_radius_f(m1);
    z1 = __fmul_rn(r, c);
    z2 = __fmul_rn(r, s);
}

// ------------------------------------------------------- float-float ----
// Error-free sum (Knuth TwoSum); the _rn intrinsics keep the compiler from
// contracting or reordering the operations.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// {hi, lo} + (dhi + dlo), renormalised.
__device__ __forceinline__ float2 ff_add(float2 a, float dhi, float dlo) {
    float s, e;
    two_sum(a.x, dhi, s, e);
    const float t = __fadd_rn(__fadd_rn(a.y, dlo), e);
    const float hi = __fadd_rn(s, t);
    return make_float2(hi, __fsub_rn(t, __fsub_rn(hi, s)));
}

// ----------------------------------------------------------- V' source ----
// R:1923-1930 lookup: fidx = (x - tmin)*dinv, idx = int(fidx) clamped to
// [0, n-2], frac = fidx - idx NOT clamped (linear extrapolation outside).
// Clamping in floating point first gives the same idx as trunc-then-clamp and
// maps NaN to 0, as the x86 reference does (cvttsd2si -> INT64_MIN -> 0).
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rn_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rn_fma(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename R>
__device__ __forceinline__ R lerp_table(const R* __restrict__ t, R tmin, R dinv, int last, R x) {
    const R fidx = rn_mul(rn_sub(x, tmin), dinv);
    R c = fidx > R(0) ? fidx : R(0);
    c = c < R(last) ? c : R(last);
    const int idx = (int)c;
    const R frac = rn_sub(fidx, R(idx));
    const R a = t[idx];
    return rn_fma(frac, rn_sub(t[idx + 1], a), a);
}

// Polynomial V'(x) = c1 x + c2 x^2 + c3 x^3 (zero-coupling inline V', R:2228:
// dV = lam*ph*ph*ph - mphi_sq*ph, evaluated in that order).
template <typename R>
__device__ __forceinline__ R poly_vprime(R c1, R c2, R c3, R x) {
    const R d = rn_fma(rn_mul(rn_mul(c3, x), x), x, rn_mul(c1, x));
    return c2 != R(0) ? rn_fma(rn_mul(c2, x), x, d) : d;
}

// ------------------------------------------------------------ storages ----
// F64: double.  F32: float with the reference's mixed arithmetic.  F32C:
// float2 {hi, lo} with value hi + lo (a 48-bit significand in 8 bytes).
__device__ __forceinline__ float2 split_f32c(double v) {
    float hi = __double2float_rn(v);
    float lo = __double2float_rn(v - (double)hi);
    return make_float2(hi, lo);
}
__device__ __forceinline__ double join_f32c(float2 v) { return (double)v.x + (double)v.y; }

}  // namespace tipt
