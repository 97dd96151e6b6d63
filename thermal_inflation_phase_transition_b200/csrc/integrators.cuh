// Alternative integrators (BAOAB, overdamped Euler-Maruyama): parameters and
// the per-site compensated-FP32 arithmetic shared by the generic kernels
// (integrators.cu) and the marching kernel (rk2_march.cu), so both give the
// same bits.  Reference: R:1974-2193 (real), C:2223-2528 (complex).
#pragma once

#include "rk2_complex.cuh"

namespace tipt {

enum { kOD = 0, kBA1 = 1, kBA2 = 2 };

struct AltParams {
    const void* f[4];  // real: phi, pi; complex: phi1, phi2, pi1, pi2
    void* o[4];
    int n0, n1, n2;
    double h, dto, inv_dx2, inv_mu2, inv_a2, c1, c2, ns;
    uint64_t step, seed;
    ComplexStageParams v;  // V' source, Z_N and eps terms (the force fields only)
};

__device__ __forceinline__ float vprime_alt_f(const ComplexStageParams& v, const float* s_tab,
                                              float x) {
    if (v.vkind == TIPT_VP_POLY)
        return poly_vprime<float>((float)v.c1, (float)v.c2, (float)v.c3, x);
    if (v.table_in_smem) return lerp_table<float>(s_tab, (float)v.tmin, (float)v.dinv, v.npts - 2, x);
    return (float)lerp_table<double>(v.table, v.tmin, v.dinv, v.npts - 2, (double)x);
}

// a + h*b as float-float (h split into hh + hl), the product error kept.
__device__ __forceinline__ void ff_axpy(float ah, float al, float hh, float hl, float bh, float bl,
                                        float& oh, float& ol) {
    const float d_hi = __fmul_rn(hh, bh);
    const float d_lo = __fadd_rn(__fmaf_rn(hh, bh, -d_hi), __fmaf_rn(hh, bl, __fmul_rn(hl, bh)));
    ff_add(ah, al, d_hi, d_lo, oh, ol);
}

// One site of the real-field step in compensated FP32 from the stencil sums of
// phi (dh = sum (hi_n - hi_c), dl = fma(-6, lo_c, sum lo_n), reference order),
// its centre (ch, cl), vp = V'(ch + cl), the noise z and pi at the site (the
// BAOAB passes).  Outputs: overdamped phi' -> (ah, al); BAOAB pass 1 phi'' ->
// (ah, al) and pi'' -> (bh, bl); pass 2 pi''' -> (bh, bl).
template <int MODE>
__device__ __forceinline__ void alt_real_site_f32c(const AltParams& p, float ch, float cl, float dh,
                                                   float dl, float vp, float z, float vh, float vl,
                                                   float& ah, float& al, float& bh, float& bl) {
    const float lap = __fmul_rn(__fadd_rn(dh, dl), (float)p.inv_dx2);
    const float F = __fsub_rn(__fmul_rn((float)p.inv_a2, lap), __fmul_rn(vp, (float)p.inv_mu2));
    if constexpr (MODE == kOD) {
        ff_add(ch, cl, __fmaf_rn((float)p.dto, F, __fmul_rn((float)p.ns, z)), 0.0f, ah, al);
    } else {
        const float h = (float)p.h, hlo = (float)(p.h - (double)h);
        if constexpr (MODE == kBA1) {
            ff_add(vh, vl, __fmul_rn(h, F), 0.0f, vh, vl);   // pi'
            float fh, fl;
            ff_axpy(ch, cl, h, hlo, vh, vl, fh, fl);          // phi'
            const float c1h = (float)p.c1, c1l = (float)(p.c1 - (double)c1h);
            const float ph_ = __fmul_rn(c1h, vh);
            const float pl_ = __fadd_rn(__fmaf_rn(c1h, vh, -ph_),
                                        __fmaf_rn(c1h, vl, __fmul_rn(c1l, vh)));
            ff_add(ph_, pl_, __fmul_rn((float)p.c2, z), 0.0f, bh, bl);  // pi''
            ff_axpy(fh, fl, h, hlo, bh, bl, ah, al);                    // phi''
        } else {
            ff_add(vh, vl, __fmul_rn(h, F), 0.0f, bh, bl);
        }
    }
}

}  // namespace tipt
