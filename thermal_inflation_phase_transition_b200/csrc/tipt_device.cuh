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

// ----------------------------------------------------------- V' source ----
// R:1923-1930 lookup: fidx = (x - tmin)*dinv, idx = int(fidx) clamped to
// [0, n-2], frac = fidx - idx NOT clamped (linear extrapolation outside).
// Clamping in floating point first gives the same idx as trunc-then-clamp and
// maps NaN to 0, as the x86 reference does (cvttsd2si -> INT64_MIN -> 0).
template <typename R>
__device__ __forceinline__ R lerp_table(const R* __restrict__ t, R tmin, R dinv, int last, R x) {
    R fidx = (x - tmin) * dinv;
    R c = fidx > R(0) ? fidx : R(0);
    c = c < R(last) ? c : R(last);
    int idx = (int)c;
    R frac = fidx - R(idx);
    R a = t[idx];
    return a + frac * (t[idx + 1] - a);
}

// Polynomial V'(x) = c1 x + c2 x^2 + c3 x^3 (zero-coupling inline V', R:2228:
// dV = lam*ph*ph*ph - mphi_sq*ph, evaluated in that order).
template <typename R>
__device__ __forceinline__ R poly_vprime(R c1, R c2, R c3, R x) {
    R d = c3 * x * x * x + c1 * x;
    return c2 != R(0) ? d + c2 * x * x : d;
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
