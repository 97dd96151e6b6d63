// Device-side building blocks shared by the lattice kernels: the counter-based
// hash noise, the V' sources and the three state storages.
//
// Reference citations: R = simulation/latticeSimeRescale_numba.py,
//                      C = simulation/latticeSimComplex_numba.py.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "tipt.h"

namespace tipt {

constexpr uint64_t kPass2Mul = 73856093ull;   // R:2518 (pass 2 / midpoint)
constexpr uint64_t kPass4Mul = 19349669ull;   // R:2643 (pass 4)
constexpr uint64_t kSeedStride = 0x9E3779B97F4A7C15ull;
constexpr double kTwoPiLit = 6.283185307179586;  // literal of R:2520

// Order-preserving integer code of a float (unsigned comparison = float order).
__device__ __forceinline__ unsigned int ord_code(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Per-thread running range of the values a launch writes.  A value that FP32
// cannot hold exactly is folded as the pair (rounded down, rounded up), so the
// range always encloses the values written: a host test `lo < t_lo` or
// `hi > t_hi` against a wider-precision bound then never misses a value just
// outside it.  Values beyond the FP32 range count as non-finite.
struct RangeAcc {
    float lo, hi;
    unsigned int bad;
    __device__ __forceinline__ RangeAcc() : lo(INFINITY), hi(-INFINITY), bad(0u) {}
    __device__ __forceinline__ void fold(float v) { fold(v, v); }
    // vd <= exact value <= vu
    __device__ __forceinline__ void fold(float vd, float vu) {
        lo = fminf(lo, vd);
        hi = fmaxf(hi, vu);
        bad |= !(vd >= -3.402823466e38f && vu <= 3.402823466e38f);   // NaN or infinite
    }
    // an FP64 value
    __device__ __forceinline__ void fold_d(double v) {
        fold(__double2float_rd(v), __double2float_ru(v));
    }
    // a compensated value hi + lo: the directed FP32 sums round the exact sum
    // down and up
    __device__ __forceinline__ void fold_ff(float h, float l) {
        fold(__fadd_rd(h, l), __fadd_ru(h, l));
    }
    // Reduction over the warp's active lanes (lanes that left early are not
    // waited for); the lowest active lane folds it into range[0..2].
    __device__ __forceinline__ void flush(unsigned int* range) {
        const unsigned int m = __activemask();
        const unsigned int l = __reduce_min_sync(m, ord_code(lo));
        const unsigned int h = __reduce_max_sync(m, ord_code(hi));
        const unsigned int b = __reduce_or_sync(m, bad);
        if ((int)(threadIdx.x & 31) == __ffs(m) - 1) {
            atomicMin(&range[0], l);
            atomicMax(&range[1], h);
            if (b) atomicOr(&range[2], 1u);
        }
    }
};

// Block 0, thread 0 resets three range words for the following launch.
__device__ __forceinline__ void reset_range_words(unsigned int* next) {
    if (next && blockIdx.x == 0 && threadIdx.x == 0) {
        next[0] = 0xFFFFFFFFu;
        next[1] = 0u;
        next[2] = 0u;
    }
}

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
    // the pass multipliers are 32-bit; a 32-bit site then needs one wide multiply
    const uint64_t sm = (site >> 32) == 0 && (mul >> 32) == 0
                            ? (uint64_t)(uint32_t)site * (uint64_t)(uint32_t)mul
                            : site * mul;
    return (sm ^ step) + seed * kSeedStride;
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

// ------------------------------------------------ FP32 lane vectors ----
// The compensated-FP32 arithmetic is written once for a "lane vector" V: a
// float (one site) or a float2 (two sites in the two lanes of Blackwell's
// packed FP32x2 instructions).  The packed intrinsics round each component
// exactly as the scalar ones, so both forms give identical bits.
__device__ __forceinline__ float v_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float v_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float v_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float v_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float v_splat(float x, float) { return x; }

__device__ __forceinline__ float2 v_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as fma(b, -1, a): exact product, one rounding -- bitwise a - b
__device__ __forceinline__ float2 v_sub(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ float2 v_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 v_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 v_splat(float x, float2) { return make_float2(x, x); }

template <typename V>
__device__ __forceinline__ V vs(float x) { return v_splat(x, V{}); }
__device__ __forceinline__ float v_neg(float a) { return -a; }
__device__ __forceinline__ float2 v_neg(float2 a) { return make_float2(-a.x, -a.y); }

// FP32 Box-Muller for the compensated-FP32 storage.  The hash is the same
// integer computation; only the Gaussian transform runs in FP32, from the
// 53-bit integers m1, m2 (u = m * 2^-53):
//  * log(u1), from the halves h1 = m1 >> 32 (< 2^21) and l1 = m1 mod 2^32: the
//    atanh series of log(1 + g), g = u1 - 1 formed exactly from the halves,
//    for u1 >= 1/2; the hardware base-2 logarithm for u1 < 1/2 (neg2_log_u1
//    below, which returns v = -2 log(u1), the factor folded into the last
//    operation of each branch: an exact scaling by -2).
//    The reference's clamp u1 >= 1e-12 is applied to the FP32 value of u1.
//  * the angle 2 pi u2, from the top 31 bits t2 of m2 (u2 = t2 2^-31 to within
//    2^-31, an angle error below 3e-9): cos alone (real field) by the nearest
//    half turn, x in [-pi/2, pi/2] and the Taylor series of cos to x^12
//    (truncated below 7e-9); cos and sin (complex field) by the nearest quarter
//    turn, x in [-pi/4, pi/4] and the series of sin (to x^9) and cos (to x^10),
//    truncated below 3e-9.
//  * sqrt via rsqrt and one Newton step.
// The absolute error of z against the FP64 reference value is a few 1e-7.
//
// hash_words: the three words of the hash the FP32 transform reads.  t2 = bits
// 33..63 of the last product, which the final x ^= x >> 31 of R:2334 leaves
// unchanged (it alters bits 0..32 only), so that step is skipped for m2.
__device__ __forceinline__ void hash_words(uint64_t x, uint32_t& h1, uint32_t& l1, uint32_t& t2) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x = x ^ (x >> 31);
    const uint64_t m1 = x >> 11;
    // (y ^ C) ^ ((y ^ C) >> 30) = y ^ (y >> 30) ^ (C ^ (C >> 30)): one xor fewer
    constexpr uint64_t kC = 0x9E3779B97F4A7C15ull, kCs = kC ^ (kC >> 30);
    x = x * 0x2545F4914F6CDD1Dull;
    x = (x ^ (x >> 30) ^ kCs) * 0xBF58476D1CE4E5B9ull;
    h1 = (uint32_t)(m1 >> 32);
    l1 = (uint32_t)m1;
    t2 = (uint32_t)(x >> 33);
}


// -2 log(u1) for one lane from the halves h, l of m1 (u1 = m1 2^-53):
//  * u1 >= 1/2: g = u1 - 1 = (h - 2^21) 2^-21 + l 2^-53 (exact to 2^-45), and
//    log(1 + g) = 2 atanh(s), s = g / (2 + g) in [-1/3, 0], summed as
//    2 s (1 + s^2/3 + ... + s^12/13) (the atanh series, truncated below 1e-8);
//  * u1 < 1/2: log2(u1) ln 2 with the hardware base-2 logarithm (lg2.approx;
//    |log2 u1| >= 1 there, so its absolute error of about 2^-22 is a relative
//    error below 2e-7), u1 first clamped to 1e-12 (R:2336).
// Both are formed and one is selected, so the lanes of a warp do not diverge.
constexpr float kLn2 = 0.693147182464599609375f;     // ln 2 rounded to FP32
constexpr float kNeg2Ln2 = -2.0f * kLn2;             // exact

__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The arithmetic of neg2_log_u1 in lane vectors (one or two lanes; the packed
// instructions round each lane as the scalar ones, so both give the same bits).
template <typename V>
__device__ __forceinline__ V neg2_log_u1_v(V hf, V lo) {
    const V g = v_fma(v_sub(hf, vs<V>(0x1p21f)), vs<V>(0x1p-21f), lo);
    const V d = v_add(vs<V>(2.0f), g);
    V r;
    if constexpr (sizeof(V) == 4) r = rcp_approx(d);
    else r = make_float2(rcp_approx(d.x), rcp_approx(d.y));
    const V s = v_mul(g, r);
    const V w = v_mul(s, s);
    V poly = v_fma(w, vs<V>(1.0f / 13.0f), vs<V>(1.0f / 11.0f));
    poly = v_fma(w, poly, vs<V>(1.0f / 9.0f));
    poly = v_fma(w, poly, vs<V>(1.0f / 7.0f));
    poly = v_fma(w, poly, vs<V>(1.0f / 5.0f));
    poly = v_fma(w, poly, vs<V>(1.0f / 3.0f));
    poly = v_mul(w, poly);
    const V m4s = v_mul(s, vs<V>(-4.0f));
    return v_fma(m4s, poly, m4s);  // -2 log(1 + g): the u1 >= 1/2 branch
}

// -2 log(u1) of the u1 < 1/2 branch for one lane from u1 in FP32
__device__ __forceinline__ float neg2_log_far(float u) {
    return __fmul_rn(lg2_approx(fmaxf(u, 1e-12f)), kNeg2Ln2);
}

__device__ __forceinline__ float neg2_log_u1(uint32_t h, uint32_t l) {
    const float lo = __fmul_rn((float)l, 0x1p-53f);
    const float hf = (float)h;  // exact: h < 2^21
    const float near = neg2_log_u1_v<float>(hf, lo);
    const float far = neg2_log_far(__fmaf_rn(hf, 0x1p-21f, lo));
    return h >= (1u << 20) ? near : far;
}

// neg2_log_u1 for two keys in the lanes of a float2.
__device__ __forceinline__ float2 neg2_log_u1_2(uint32_t ha, uint32_t la, uint32_t hb,
                                                uint32_t lb) {
    const float2 lo = v_mul(make_float2((float)la, (float)lb), vs<float2>(0x1p-53f));
    const float2 hf = make_float2((float)ha, (float)hb);
    const float2 near = neg2_log_u1_v<float2>(hf, lo);
    const float2 u = v_fma(hf, vs<float2>(0x1p-21f), lo);
    return make_float2(ha >= (1u << 20) ? near.x : neg2_log_far(u.x),
                       hb >= (1u << 20) ? near.y : neg2_log_far(u.y));
}

// Quarter-turn reduction of 2 pi u2 (u2 = t 2^-31): q = round(4 u2) and the
// remainder x = 2 pi u2 - q pi/2 in [-pi/4, pi/4].  The remainder
// rh = t - q 2^29 is the low 29 bits of t read as a signed number, so
// (int)(t << 3) = 8 rh exactly; its conversion is 8 (float)rh and the constant
// carries the 2^-3, so x is bitwise (float)rh (pi/2) 2^-29.
__device__ __forceinline__ void angle_reduce(uint32_t t, uint32_t& q, float& x) {
    q = (t + (1u << 28)) >> 29;                        // nearest multiple of 2^29
    const int r8 = (int)(t << 3);                      // 8 rh, |rh| <= 2^28
    x = __fmul_rn((float)r8, 0x1.921fb6p-32f /* (pi/2) 2^-29 2^-3, rounded to FP32 */);
}

__device__ __forceinline__ void sincos_series1(float x, float& sn, float& cs) {
    const float x2 = __fmul_rn(x, x);
    float sp = __fmaf_rn(x2, 2.75573192e-6f, -1.98412698e-4f);   // 1/9!, -1/7!
    sp = __fmaf_rn(x2, sp, 8.33333333e-3f);                      // 1/5!
    sp = __fmaf_rn(x2, sp, -1.66666667e-1f);                     // -1/3!
    sn = __fmaf_rn(__fmul_rn(x2, x), sp, x);
    float cp = __fmaf_rn(x2, -2.75573192e-7f, 2.48015873e-5f);   // -1/10!, 1/8!
    cp = __fmaf_rn(x2, cp, -1.38888889e-3f);                     // -1/6!
    cp = __fmaf_rn(x2, cp, 4.16666667e-2f);                      // 1/4!
    cp = __fmaf_rn(x2, cp, -0.5f);
    cs = __fmaf_rn(x2, cp, 1.0f);
}

template <typename V>
__device__ __forceinline__ void sincos_series(V x, V& sn, V& cs) {
    if constexpr (sizeof(V) == 4) {
        sincos_series1(x, sn, cs);
    } else {
        sincos_series1(x.x, sn.x, cs.x);
        sincos_series1(x.y, sn.y, cs.y);
    }
}

// rotate (cos x, sin x) by q quarter turns -> (cos, sin) of the full angle
__device__ __forceinline__ void quarter_turn(uint32_t q, float sn, float cs, float& c, float& s) {
    const uint32_t qq = q & 3u;
    const float a = (qq & 1u) ? sn : cs;
    const float b = (qq & 1u) ? cs : sn;
    c = (qq == 1u || qq == 2u) ? -a : a;
    s = (qq >= 2u) ? -b : b;
}

// sqrt(v) for v = -2 log(u1) > 0
template <typename V>
__device__ __forceinline__ V radius_from_v(V v) {
    V y;
    if constexpr (sizeof(V) == 4) y = rsqrtf(v);
    else y = make_float2(rsqrtf(v.x), rsqrtf(v.y));
    const V r = v_mul(v, y);
    return v_fma(v_mul(vs<V>(0.5f), y), v_fma(v_neg(r), r, v), r);  // one Newton step
}

// cos(2 pi u2) alone (the real field draws only the cos branch): half-turn
// reduction 2 u2 = q + x/pi with q = round(2 u2) in {0, 1, 2} and
// x in [-pi/2, pi/2], cos = (-1)^q cos x.  Returns x and a word whose bit 31 is
// q's parity (the other bits are not defined).  As in angle_reduce, the
// remainder rh = t - q 2^30 is the low 30 bits of t read as a signed number:
// (int)(t << 2) = 4 rh, and the constant carries the 2^-2.
__device__ __forceinline__ void half_turn_reduce(uint32_t t, uint32_t& sign, float& x) {
    const int r4 = (int)(t << 2);                      // 4 rh, |rh| <= 2^29
    x = __fmul_rn((float)r4, 0x1.921fb6p-31f /* pi 2^-30 2^-2, rounded to FP32 */);
    sign = (t + (1u << 29)) << 1;                      // bit 31 = bit 30 of t + 2^29 = q & 1
}

template <typename V>
__device__ __forceinline__ V cos_series(V x) {
    const V x2 = v_mul(x, x);
    V c = v_fma(x2, vs<V>(2.08767570e-9f), vs<V>(-2.75573192e-7f));  // 1/12!, -1/10!
    c = v_fma(x2, c, vs<V>(2.48015873e-5f));                         // 1/8!
    c = v_fma(x2, c, vs<V>(-1.38888889e-3f));                        // -1/6!
    c = v_fma(x2, c, vs<V>(4.16666667e-2f));                         // 1/4!
    c = v_fma(x2, c, vs<V>(-0.5f));
    return v_fma(x2, c, vs<V>(1.0f));
}

// v with its sign flipped where bit 31 of `sign` is set (the other bits of
// `sign` are ignored)
__device__ __forceinline__ float flip_sign(float v, uint32_t sign) {
    return __uint_as_float(__float_as_uint(v) ^ (sign & 0x80000000u));
}

// z (cos branch) for one key, FP32.
__device__ __forceinline__ float gauss_cos_f(uint64_t key) {
    uint32_t h1, l1, t2, sg;
    hash_words(key, h1, l1, t2);
    float x;
    const float v = neg2_log_u1(h1, l1);
    half_turn_reduce(t2, sg, x);
    return __fmul_rn(radius_from_v<float>(v), flip_sign(cos_series<float>(x), sg));
}

// z for two keys in the two lanes of a float2 (bitwise the same as two calls
// of gauss_cos_f).
__device__ __forceinline__ float2 gauss_cos_f2(uint64_t key0, uint64_t key1) {
    uint32_t h1a, l1a, t2a, h1b, l1b, t2b, sa, sb;
    hash_words(key0, h1a, l1a, t2a);
    hash_words(key1, h1b, l1b, t2b);
    float xa, xb;
    const float2 v = neg2_log_u1_2(h1a, l1a, h1b, l1b);
    half_turn_reduce(t2a, sa, xa);
    half_turn_reduce(t2b, sb, xb);
    const float2 cx = cos_series<float2>(make_float2(xa, xb));
    const float2 c = make_float2(flip_sign(cx.x, sa), flip_sign(cx.y, sb));
    return v_mul(radius_from_v<float2>(v), c);
}

// (z1, z2) = r (cos, sin) for one key (complex field, one pair per site).
__device__ __forceinline__ void gauss_pair_f(uint64_t key, float& z1, float& z2) {
    uint32_t h1, l1, t2, q;
    hash_words(key, h1, l1, t2);
    float x, sn, cs, c, s;
    const float v = neg2_log_u1(h1, l1);
    angle_reduce(t2, q, x);
    sincos_series<float>(x, sn, cs);
    quarter_turn(q, sn, cs, c, s);
    const float r = radius_from_v<float>(v);
    z1 = __fmul_rn(r, c);
    z2 = __fmul_rn(r, s);
}

// (z1, z2) pairs for two keys in the lanes of float2s (bitwise the same as two
// calls of gauss_pair_f).
__device__ __forceinline__ void gauss_pair_f2(uint64_t key0, uint64_t key1, float2& z1,
                                              float2& z2) {
    uint32_t h1a, l1a, t2a, h1b, l1b, t2b, qa, qb;
    hash_words(key0, h1a, l1a, t2a);
    hash_words(key1, h1b, l1b, t2b);
    float xa, xb;
    const float2 v = neg2_log_u1_2(h1a, l1a, h1b, l1b);
    angle_reduce(t2a, qa, xa);
    angle_reduce(t2b, qb, xb);
    float2 sn, cs;
    sincos_series<float2>(make_float2(xa, xb), sn, cs);
    float2 c, s;
    quarter_turn(qa, sn.x, cs.x, c.x, s.x);
    quarter_turn(qb, sn.y, cs.y, c.y, s.y);
    const float2 r = radius_from_v<float2>(v);
    z1 = v_mul(r, c);
    z2 = v_mul(r, s);
}

// ------------------------------------------------------- float-float ----
// Error-free sum (Knuth TwoSum) and a renormalised float-float add, in lane
// vectors; every operation is an explicit round-to-nearest intrinsic.

template <typename V>
__device__ __forceinline__ void two_sum(V a, V b, V& s, V& e) {
    s = v_add(a, b);
    const V bb = v_sub(s, a);
    e = v_add(v_sub(a, v_sub(s, bb)), v_sub(b, bb));
}

// (hi, lo) + (dhi + dlo), renormalised.
template <typename V>
__device__ __forceinline__ void ff_add(V ahi, V alo, V dhi, V dlo, V& hi, V& lo) {
    V s, e;
    two_sum(ahi, dhi, s, e);
    const V t = v_add(v_add(alo, dlo), e);
    hi = v_add(s, t);
    lo = v_sub(t, v_sub(hi, s));
}

// (hi, lo) + d for a single FP32 increment d, renormalised.
template <typename V>
__device__ __forceinline__ void ff_add1(V ahi, V alo, V d, V& hi, V& lo) {
    V s, e;
    two_sum(ahi, d, s, e);
    const V t = v_add(alo, e);
    hi = v_add(s, t);
    lo = v_sub(t, v_sub(hi, s));
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

// FP32 lookup in a V' row staged in shared memory, for a lane vector of
// fractional indices fidx = (x - tmin) dinv: the lerp_table rule lane by lane
// (index clamped to [0, last], fraction unclamped).
__device__ __forceinline__ float vlane(float v, int) { return v; }
__device__ __forceinline__ float vlane(float2 v, int l) { return l ? v.y : v.x; }
__device__ __forceinline__ void vset(float& v, int, float x) { v = x; }
__device__ __forceinline__ void vset(float2& v, int l, float x) {
    if (l) v.y = x;
    else v.x = x;
}

__device__ __forceinline__ float v_add_rz(float a, float b) { return __fadd_rz(a, b); }
__device__ __forceinline__ float2 v_add_rz(float2 a, float2 b) { return __fadd2_rz(a, b); }

template <typename V>
__device__ __forceinline__ V lerp_table_f32(const float* s_tab, V fidx, float last) {
    constexpr int NL = sizeof(V) / sizeof(float);
    V c;
#pragma unroll
    for (int l = 0; l < NL; ++l) vset(c, l, fminf(fmaxf(vlane(fidx, l), 0.0f), last));
    // c in [0, last]: c + 2^23 rounded toward zero is trunc(c) + 2^23 exactly, so
    // its low mantissa bits are the index and subtracting 2^23 gives trunc(c)
    const V t = v_add_rz(c, vs<V>(0x1p23f));
    V a, b;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        const int idx = (int)(__float_as_uint(vlane(t, l)) - 0x4B000000u);
        vset(a, l, s_tab[idx]);
        vset(b, l, s_tab[idx + 1]);
    }
    const V fi = v_sub(t, vs<V>(0x1p23f));
    return v_fma(v_sub(fidx, fi), v_sub(b, a), a);
}

// The same lookup from a table of (value, slope) pairs, slope[q] = v[q+1] - v[q]
// rounded to FP32 when the table is staged: one 8-byte load per lane, and the
// bits of lerp_table_f32 (its b - a is that same FP32 difference).
template <typename V>
__device__ __forceinline__ V lerp_pairs_f32(const float2* s_tab2, V fidx, float last) {
    constexpr int NL = sizeof(V) / sizeof(float);
    V c;
#pragma unroll
    for (int l = 0; l < NL; ++l) vset(c, l, fminf(fmaxf(vlane(fidx, l), 0.0f), last));
    const V t = v_add_rz(c, vs<V>(0x1p23f));
    V a, d;
#pragma unroll
    for (int l = 0; l < NL; ++l) {
        const float2 e = s_tab2[__float_as_uint(vlane(t, l)) - 0x4B000000u];
        vset(a, l, e.x);
        vset(d, l, e.y);
    }
    const V fi = v_sub(t, vs<V>(0x1p23f));
    return v_fma(v_sub(fidx, fi), d, a);
}

// Polynomial V'(x) = c1 x + c2 x^2 + c3 x^3 (zero-coupling inline V', R:2228:
// dV = lam*ph*ph*ph - mphi_sq*ph, evaluated in that order).
template <typename R>
__device__ __forceinline__ R poly_vprime(R c1, R c2, R c3, R x) {
    const R d = rn_fma(rn_mul(rn_mul(c3, x), x), x, rn_mul(c1, x));
    return c2 != R(0) ? rn_fma(rn_mul(c2, x), x, d) : d;
}

}  // namespace tipt
