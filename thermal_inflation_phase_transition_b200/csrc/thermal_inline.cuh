// The thermal one-loop V' evaluated per site, as the reference's inline form
// _vprime_inline (R:2201-2266) that rk2_fused_single_pass (R:2339-2647) calls
// or (form 1) as Vprime_field (R:1435-1485) that rk2_step / rk2_step_fused call:
//   V' = lam phi^3 - mphi^2 phi + T^4/(2 pi^2) (cb dJ_B(x_b) dx_b/dphi + cf dJ_F(x_f) dx_f/dphi),
//   x_b = sqrt(mB^2 + gb^2 phi^2/2 + (gb^2/4 + 2 gg^2/3) T^2) / T,
//   x_f = sqrt(gf^2 phi^2/2 + gfg^2 T^2/6) / T,
// dJ from the cubic splines on the uniform grid x_min + i h: inline form x
// clamped to [x_min, xhi], xhi = x_min + h nseg - 1e-12, segment
// trunc((x - x_min) * (1/h)); field form x below x_min raised to x_min, x above
// x_min + h nseg lowered to x_min + h nseg - 1e-12, segment trunc((x - x_min) / h);
// the segment clamped to [0, nseg-1] in both.
// FP64, in the reference's order of operations.
#pragma once

#include "tipt.h"

namespace tipt {

// Per-launch constants (computed on the host from tipt_thermal and T).
struct ThermalSite {
    const double* spline;  // [8][nseg]: dx^3, dx^2, dx, 1 coefficients of dJ_B, then dJ_F
    int nseg;
    int field_form;        // 1: the Vprime_field / cubic_eval_uniform clamp and segment rule
    double lam, mphi_sq, bms, gb2, gf2, gfg2, coef_b, coeff_b, coeff_f;
    double x_min, h, inv_hy, xhi, xtop;
    double T, T2, pref;
};

inline ThermalSite thermal_site(const tipt_thermal& t, double T) {
    ThermalSite s;
    s.spline = t.spline;
    s.nseg = t.nseg;
    s.lam = t.lam;
    s.mphi_sq = t.mphi * t.mphi;
    s.bms = t.boson_mass_sq;
    s.gb2 = t.boson_coupling * t.boson_coupling;
    const double gg2 = t.boson_gauge_coupling * t.boson_gauge_coupling;
    s.gf2 = t.fermion_coupling * t.fermion_coupling;
    s.gfg2 = t.fermion_gauge_coupling * t.fermion_gauge_coupling;
    s.coef_b = 0.25 * s.gb2 + (2.0 / 3.0) * gg2;  // R:2376
    s.coeff_b = t.coeff_b;
    s.coeff_f = t.coeff_f;
    s.x_min = t.x_min;
    s.h = t.h;
    s.inv_hy = 1.0 / t.h;                       // R:452
    s.xhi = t.x_min + t.h * t.nseg - 1e-12;     // R:453
    s.xtop = t.x_min + t.h * t.nseg;            // R:1467-1468
    s.field_form = t.form == 1;
    s.T = T;
    s.T2 = T * T;
    s.pref = s.T2 * s.T2 / (2.0 * 3.141592653589793 * 3.141592653589793);
    return s;
}

__device__ __forceinline__ double thermal_dj(const double* c, const ThermalSite& s, double x) {
    const int nseg = s.nseg;
    double xc = x;
    int si;
    if (s.field_form) {  // R:1464-1473, R:1418-1424
        if (xc < s.x_min) xc = s.x_min;
        else if (xc > s.xtop) xc = s.xtop - 1e-12;
        si = (int)((xc - s.x_min) / s.h);
    } else {             // R:2238-2248
        if (xc < s.x_min) xc = s.x_min;
        else if (xc > s.xhi) xc = s.xhi;
        si = (int)((xc - s.x_min) * s.inv_hy);
    }
    si = si < 0 ? 0 : (si >= nseg ? nseg - 1 : si);
    const double d = xc - (s.x_min + si * s.h);
    return ((c[si] * d + c[nseg + si]) * d + c[2 * nseg + si]) * d + c[3 * nseg + si];
}

__device__ __forceinline__ double thermal_vprime_inline(const ThermalSite& s, double ph) {
    double dV = s.lam * ph * ph * ph - s.mphi_sq * ph;
    const double xb_sq = s.bms + 0.5 * s.gb2 * ph * ph + s.coef_b * s.T2;
    const double xb = xb_sq > 0.0 ? sqrt(xb_sq) / s.T : 0.0;
    const double xf_sq = 0.5 * s.gf2 * ph * ph + (1.0 / 6.0) * s.gfg2 * s.T2;
    const double xf = xf_sq > 0.0 ? sqrt(xf_sq) / s.T : 0.0;
    const double dJb = thermal_dj(s.spline, s, xb);
    const double dJf = thermal_dj(s.spline + 4 * s.nseg, s, xf);
    const double dxb = 0.5 * s.gb2 * ph / (s.T2 * fmax(xb, 1e-20));
    const double dxf = 0.5 * s.gf2 * ph / (s.T2 * fmax(xf, 1e-20));
    dV += s.pref * (s.coeff_b * dJb * dxb + s.coeff_f * dJf * dxf);
    return dV;
}

}  // namespace tipt
