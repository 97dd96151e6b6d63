// Complex-field (Phi = phi1 + i phi2) per-site arithmetic shared by the generic
// stage kernel (rk2_complex.cu) and the marching kernel (rk2_march.cu):
// C:2067-2215 rk2_step_table, fused into one midpoint stage as for the real
// field (phi~_a = phi_a + h1 pi_a is pointwise).
#pragma once

#include "rk2_real.cuh"

namespace tipt {

// FP32 constants of a compensated-FP32 complex stage as lane pairs, rounded
// once on the host from the FP64 parameters (set_complex_f32): the per-site
// arithmetic then converts nothing.
struct ComplexF32 {
    float2 h1, h2h, h2l;       // h2 = h2h + h2l
    float2 lsc;                // inv_a2 inv_dx2
    float2 neg_eta, neg_imu2;
    float2 ns;                 // hash noise amplitude
};

struct ComplexStageParams {
    const void* f[4];   // phi1, phi2, pi1, pi2
    void* o[4];
    int n0, n1, n2;
    double h1, h2, inv_dx2, eta, inv_mu2, inv_a2;
    const void* noise1;
    const void* noise2;
    double ns_eff, nfac;
    uint64_t step, mul, seed;
    double zn_n, zn_dv, zn_active, eps4;
    // V'(rho) source (1-D table or polynomial)
    int vkind, npts;
    const double* table;
    double tmin, dinv;
    double c1, c2, c3;
    int table_in_smem;
    ThermalSite th;  // TIPT_VP_THERMAL: the inline thermal V'(rho) at T
    // Range of the new |Phi| (optional, the complex loop's per-step rho check,
    // C:4263-4288): as RealStageParams::range, folded from rho = sqrt(phi1^2 +
    // phi2^2) of the values written (FP32 for the compensated and float32
    // storages, FP64 rounded to FP32 for FP64).
    unsigned int* range;
    unsigned int* range_next;
    ComplexF32 k2;  // set by set_complex_f32 before every launch
};

__host__ __device__ inline void set_complex_f32(ComplexStageParams& p) {
    auto pr = [](float x) { return make_float2(x, x); };
    const float h2h = (float)p.h2;
    p.k2.h1 = pr((float)p.h1);
    p.k2.h2h = pr(h2h);
    p.k2.h2l = pr((float)(p.h2 - (double)h2h));
    p.k2.lsc = pr((float)(p.inv_a2 * p.inv_dx2));
    p.k2.neg_eta = pr((float)(-p.eta));
    p.k2.neg_imu2 = pr((float)(-p.inv_mu2));
    p.k2.ns = pr((float)p.ns_eff);
}

// rho of the values written, as the range folds it.  float32 storage: the
// FP32 value the reference's float32 arrays give.  FP64: the FP64 value,
// rounded outward to FP32.  Compensated FP32 (a = ah + al, b = bh + bl): FP32
// bounds from directed roundings, |ah| - |al| <= |a| <= |ah| + |al|, so the
// folded range encloses the exact |Phi| of every site written.
__device__ __forceinline__ float rho_f32(float a, float b) {
    return __fsqrt_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)));
}
__device__ __forceinline__ void fold_rho_f64(RangeAcc& r, double a, double b) {
    r.fold_d(__dsqrt_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b))));
}
__device__ __forceinline__ void fold_rho_ff(RangeAcc& r, float ah, float al, float bh, float bl) {
    const float au = __fadd_ru(fabsf(ah), fabsf(al)), bu = __fadd_ru(fabsf(bh), fabsf(bl));
    const float ad = fmaxf(__fsub_rd(fabsf(ah), fabsf(al)), 0.0f);
    const float bd = fmaxf(__fsub_rd(fabsf(bh), fabsf(bl)), 0.0f);
    r.fold(__fsqrt_rd(__fadd_rd(__fmul_rd(ad, ad), __fmul_rd(bd, bd))),
           __fsqrt_ru(__fadd_ru(__fmul_ru(au, au), __fmul_ru(bu, bu))));
}

// C:2137-2158 projection + Z_N (reference form), then eps*Re(Phi^4) whose
// gradient is 4 eps (p1^3 - 3 p1 p2^2, 3 p1^2 p2 - p2^3).  FP64 (and the
// reference float32 mode's FP64 arithmetic).
// TH = false compiles the thermal branch out (callers that never take it).
template <typename R, bool TH = true>
__device__ __forceinline__ void complex_force(const ComplexStageParams& p, const R* tab, R tmin,
                                              R dinv, R p1, R p2, R& d1, R& d2) {
    R rho = sqrt(p1 * p1 + p2 * p2);
    R rho_safe = rho > R(1e-30) ? rho : R(1e-30);
    R dvdr, a, b;
    if (TH && p.vkind == TIPT_VP_THERMAL) {
        // C:2605-2680 _vprime_complex_inline: V'(rho_safe) times phi_a * (1 / rho_safe)
        dvdr = (R)thermal_vprime_inline(p.th, (double)rho_safe);
        const R inv_rho = R(1) / rho_safe;
        a = dvdr * p1 * inv_rho;
        b = dvdr * p2 * inv_rho;
    } else {
        if (p.vkind == TIPT_VP_POLY) dvdr = poly_vprime<R>((R)p.c1, (R)p.c2, (R)p.c3, rho);
        else dvdr = lerp_table<R>(tab, tmin, dinv, p.npts - 2, rho);
        a = dvdr * p1 / rho_safe;
        b = dvdr * p2 / rho_safe;
    }
    if (p.zn_active > 0.5 && p.zn_n > 0.5 && rho > R(1e-20)) {
        R th = atan2(p2, p1);
        R sn = sin((R)p.zn_n * th);
        R ir = R(1) / rho_safe;
        R ir2 = ir * ir;
        a += -(R)p.zn_n * (R)p.zn_dv * sn * p2 * ir2;
        b += (R)p.zn_n * (R)p.zn_dv * sn * p1 * ir2;
    }
    if (p.eps4 != 0.0) {
        const R e4 = R(4) * (R)p.eps4;
        a += e4 * (p1 * p1 * p1 - R(3) * p1 * p2 * p2);
        b += e4 * (R(3) * p1 * p1 * p2 - p2 * p2 * p2);
    }
    d1 = a;
    d2 = b;
}

// ------------------------------------------------ compensated FP32, lanes ----
// One site (V = float) or two sites in the lanes of the packed FP32x2
// instructions (V = float2); every operation is an explicit round-to-nearest
// intrinsic, lane by lane the same, so the generic and marching kernels agree
// bitwise.  Used when Z_N is off and V'(rho) is a polynomial or a table staged
// in shared memory as FP32.

// 1/sqrt(x) for x > 0: the hardware approximation refined by one Newton-Raphson
// step, y (1 + (1 - x y^2) / 2).
__device__ __forceinline__ float rsqrt_nr(float x) {
    const float y = rsqrtf(x);
    const float e = __fmaf_rn(-__fmul_rn(x, y), y, 1.0f);
    return __fmaf_rn(__fmul_rn(0.5f, y), e, y);
}
__device__ __forceinline__ float v_rsqrt_nr(float a) { return rsqrt_nr(a); }
__device__ __forceinline__ float2 v_rsqrt_nr(float2 a) {
    return make_float2(rsqrt_nr(a.x), rsqrt_nr(a.y));
}
__device__ __forceinline__ float v_atleast(float a, float m) { return a > m ? a : m; }
__device__ __forceinline__ float2 v_atleast(float2 a, float m) {
    return make_float2(a.x > m ? a.x : m, a.y > m ? a.y : m);
}

// V'(rho) from the polynomial or the FP32 shared-memory table (R:1923-1930 rule).
template <typename V>
__device__ __forceinline__ V cvprime_v(const ComplexStageParams& p, const float* s_tab, V x,
                                       float tmin, float dinv) {
    if (p.vkind == TIPT_VP_POLY) {
        const V d = v_fma(v_mul(v_mul(vs<V>((float)p.c3), x), x), x, v_mul(vs<V>((float)p.c1), x));
        return p.c2 != 0.0 ? v_fma(v_mul(vs<V>((float)p.c2), x), x, d) : d;
    }
    // fractional index x dinv - tmin dinv (one rounding; the compensated-FP32 rule)
    return lerp_table_f32<V>(s_tab, v_fma(x, vs<V>(dinv), vs<V>(-tmin * dinv)),
                             (float)(p.npts - 2));
}

// dV/dphi_a of V(rho) + eps Re(Phi^4): V'(rho) phi_a / rho plus
// 4 eps phi1 (phi1^2 - 3 phi2^2), 4 eps phi2 (3 phi1^2 - phi2^2).  One reciprocal
// square root gives both rho = rho^2 / rho and the 1/rho of the projection;
// rho^2 is floored at 1e-36 (the reference floors rho at 1e-30, below FP32's
// range: fields with |Phi| < 1e-18 are treated as |Phi| = 1e-18).
// SRC: kCsrcAny dispatches on p at run time; kCsrcTab / kCsrcTabEps fix the
// staged-table source without / with the eps term at compile time (the same
// operations as the dispatching form's branches).
enum : int { kCsrcAny = 0, kCsrcTab = 1, kCsrcTabEps = 2 };

template <typename V, int SRC = kCsrcAny>
__device__ __forceinline__ void complex_force_v(const ComplexStageParams& p, const float* s_tab,
                                                float tmin, float dinv, V p1, V p2, V& d1,
                                                V& d2) {
    const V r2 = v_atleast(v_fma(p1, p1, v_mul(p2, p2)), 1e-36f);
    const V ri = v_rsqrt_nr(r2);
    const V rho = v_mul(r2, ri);
    V vp;
    if constexpr (SRC == kCsrcAny)
        vp = cvprime_v<V>(p, s_tab, rho, tmin, dinv);
    else  // cvprime_v's table branch
        vp = lerp_table_f32<V>(s_tab, v_fma(rho, vs<V>(dinv), vs<V>(-tmin * dinv)),
                               (float)(p.npts - 2));
    const V s = v_mul(vp, ri);
    V a = v_mul(s, p1), b = v_mul(s, p2);
    if (SRC == kCsrcTabEps || (SRC == kCsrcAny && p.eps4 != 0.0)) {
        const V e4 = vs<V>((float)(4.0 * p.eps4));
        const V q1 = v_mul(p1, p1), q2 = v_mul(p2, p2);
        a = v_fma(v_mul(e4, p1), v_fma(vs<V>(-3.0f), q2, q1), a);
        b = v_fma(v_mul(e4, p2), v_fma(vs<V>(3.0f), q1, v_neg(q2)), b);
    }
    d1 = a;
    d2 = b;
}

// Stencil sums (order ip, im, jp, jm, kp, km; dh = sum (hi_n - hi_c),
// dl = fma(-6, lo_c, sum lo_n)) and centre hi/lo of phi1, phi2, pi1, pi2.
template <typename V>
struct CplxIn {
    V dh[4], dl[4], ch[4], cl[4];
};

// The midpoint step of one site: new (hi, lo) of phi1, phi2, pi1, pi2 into
// oh[4], ol[4].  `force(q1, q2, which, d1, d2)` evaluates dV/dphi at the centre
// (which = 0) or at the midpoint (which = 1); kick[a] is the noise increment.
template <typename V, typename Force>
__device__ __forceinline__ void complex_update_f32c(const ComplexStageParams& p, const CplxIn<V>& x,
                                                    const V kick[2], Force force, V oh[4],
                                                    V ol[4]) {
    const V h1 = kvec<V>(p.k2.h1);
    const V h2h = kvec<V>(p.k2.h2h);
    const V h2l = kvec<V>(p.k2.h2l);
    // Laplacians times inv_a2 (inv_a2 inv_dx2 applied once); forces as two fused
    // multiply-adds
    const V lsc = kvec<V>(p.k2.lsc);
    const V neg_eta = kvec<V>(p.k2.neg_eta), neg_imu2 = kvec<V>(p.k2.neg_imu2);
    V lap[4], c[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        lap[f] = v_mul(v_add(x.dh[f], x.dl[f]), lsc);
        c[f] = v_add(x.ch[f], x.cl[f]);
    }
    V d1, d2;
    force(c[0], c[1], 0, d1, d2);
    const V k1[2] = {force_fma(neg_eta, neg_imu2, lap[0], c[2], d1),
                     force_fma(neg_eta, neg_imu2, lap[1], c[3], d2)};
    V t_hi[2], t_lo[2], pit[2], q[2];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        V e;
        two_sum(x.ch[2 + a], v_mul(h1, k1[a]), t_hi[a], e);
        t_lo[a] = v_add(x.cl[2 + a], e);
        pit[a] = v_add(t_hi[a], t_lo[a]);
        q[a] = v_add(x.ch[a], v_fma(h1, c[2 + a], x.cl[a]));
    }
    force(q[0], q[1], 1, d1, d2);
    const V k2[2] = {force_fma(neg_eta, neg_imu2, v_fma(h1, lap[2], lap[0]), pit[0], d1),
                     force_fma(neg_eta, neg_imu2, v_fma(h1, lap[3], lap[1]), pit[1], d2)};
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const V d_hi = v_mul(h2h, t_hi[a]);
        const V d_lo = v_add(v_fma(h2h, t_hi[a], v_neg(d_hi)), v_fma(h2h, t_lo[a], v_mul(h2l, t_hi[a])));
        ff_add(x.ch[a], x.cl[a], d_hi, d_lo, oh[a], ol[a]);
        ff_add1(x.ch[2 + a], x.cl[2 + a], v_fma(h2h, k2[a], kick[a]), oh[2 + a], ol[2 + a]);
    }
}

// Inline hash noise of one complex site: (ns z1, ns z2) from one Box-Muller pair.
__device__ __forceinline__ void complex_kick_f32c(const ComplexStageParams& p, uint64_t site,
                                                  float& k1, float& k2) {
    if (p.ns_eff == 0.0) {
        k1 = k2 = 0.0f;
        return;
    }
    float z1, z2;
    gauss_pair_f(noise_key(site, p.step, p.mul, p.seed), z1, z2);
    k1 = __fmul_rn(p.k2.ns.x, z1);
    k2 = __fmul_rn(p.k2.ns.x, z2);
}

// The same for two sites in float2 lanes (bitwise two calls of complex_kick_f32c).
__device__ __forceinline__ void complex_kick_f32c2(const ComplexStageParams& p, uint64_t s0,
                                                   uint64_t s1, float2& k1, float2& k2) {
    if (p.ns_eff == 0.0) {
        k1 = k2 = make_float2(0.0f, 0.0f);
        return;
    }
    float2 z1, z2;
    gauss_pair_f2(noise_key(s0, p.step, p.mul, p.seed), noise_key(s1, p.step, p.mul, p.seed), z1,
                  z2);
    const float2 ns = p.k2.ns;
    k1 = v_mul(ns, z1);
    k2 = v_mul(ns, z2);
}

}  // namespace tipt
