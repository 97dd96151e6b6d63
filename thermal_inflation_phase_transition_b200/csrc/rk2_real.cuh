// Real-field midpoint RK2 stage: per-site arithmetic for the three storages
// and the launch parameters shared by the generic and the marching kernels.
//
// One midpoint stage advances (phi, pi) by h2 using the midpoint state at h1
// (R:1902-1966, rk2_step_table: h1 = dt/2, h2 = dt, noise factor 1; each half
// of rk2_fused_table R:1742-1872: h1 = h2 = dt/2, noise factor 1/2).
// phi~ = phi + h1*pi depends on the site alone, so the second pass's
// Laplacian of phi~ needs only (phi, pi) on the 7-point stencil: the two
// reference passes fuse into one launch with a radius-1 halo and no scratch.
#pragma once

#include "thermal_inline.cuh"
#include "tipt_device.cuh"

namespace tipt {

struct RealStageParams {
    const void* phi;
    const void* pi;
    void* phi_out;
    void* pi_out;
    int n0, n1, n2;      // lattice extents (nx, ny, nz); n2 contiguous
    double h1, h2;       // midpoint offset, advance
    double inv_dx2, eta, inv_mu2, inv_a2;
    const void* noise;   // array noise (storage precision) or nullptr
    double ns_eff;       // hash noise amplitude incl. the 1/2 of half steps
    double nfac;         // array-noise factor (1 or 1/2)
    uint64_t step, mul, seed;
    // V' source
    int vkind;           // TIPT_VP_*
    int npts;
    const double* table; // 1-D row or 2-D [nT][npts]
    double tmin, dinv;
    int nT;
    double T_min, T_dinv, T;
    double c1, c2, c3;
    int table_in_smem;   // 1: stage (and blend) the row into dynamic smem
    // Device-resident schedule (for graph-captured step loops): when sched is
    // set, the step is s = *ctr + offset, row e = min(s, sched_len - 1) of
    // sched_cols doubles gives T = sched[cols e], the noise amplitude
    // ns_mult * sched[cols e + 1] and, with 4 columns (an expanding
    // background), eta_eff = sched[4e + 2] and inv_a2 = sched[4e + 3]; the hash
    // step is step + s.
    const double* sched;
    const unsigned long long* ctr;
    long long offset;
    long long sched_len;  // steps beyond the schedule reuse its last entry
    double ns_mult;
    int sched_cols;       // 2 (T, ns) or 4 (T, ns, eta_eff, inv_a2)
    // FP32 constants of the compensated storage as lane pairs (x = y), rounded
    // from the FP64 parameters on the host (set_f32c_pairs): the packed FP32x2
    // instructions then read them from the parameter bank.
    // lap_scale = inv_a2 inv_dx2, neg_eta = -eta, neg_imu2 = -inv_mu2 (the forces as
    // two fused multiply-adds); tmd = -tmin dinv (the table index as one).
    struct {
        float2 h1, h2h, h2l, inv_dx2, inv_a2, eta, inv_mu2, c1, c2, c3, tmin, dinv;
        float2 lap_scale, neg_eta, neg_imu2, tmd;
    } k2;
    // Planes computed: [i_begin, i_end) of the n0 planes (all planes, periodic
    // in i, when i_end = 0); the noise key's site is the array index plus
    // site_offset (a slab of a larger lattice keys by the global index).
    int i_begin, i_end;
    long long site_offset;
    ThermalSite th;  // TIPT_VP_THERMAL: the inline thermal V' at T
    // Range of the new phi (optional, the reference loop's per-step phi.min() /
    // phi.max(), R:3655-3660): the launch folds the minimum and maximum of the
    // values written (rounded outward to FP32, as order-preserving integer codes)
    // and a non-finite flag into range[0..2]; block 0 first resets
    // range_next[0..2] for the following launch.
    unsigned int* range;
    unsigned int* range_next;
    // Test of the bounded device waits (0 = off): with k > 0 the producer of
    // block 0 of the compensated-FP32 marching stage issues no copy from ring
    // position k - 1 on, so its consumers' waits for that plane expire and
    // report TIPT_ERR_TIMEOUT (tipt_test_withhold_plane arms one launch).
    int test_withhold;
};

// Block 0, thread 0 resets the range words of the following launch.
__device__ __forceinline__ void reset_next_range(const RealStageParams& p) {
    reset_range_words(p.range_next);
}

// Resolve the per-step scalars of a scheduled launch (no-op otherwise).
__device__ __forceinline__ void resolve_schedule(RealStageParams& p) {
    if (!p.sched) return;
    const unsigned long long s = *p.ctr + (unsigned long long)p.offset;
    const unsigned long long e = s < (unsigned long long)p.sched_len ? s : p.sched_len - 1;
    const double* row = p.sched + (p.sched_cols == 4 ? 4 * e : 2 * e);
    p.T = row[0];
    p.ns_eff = p.ns_mult * row[1];
    if (p.sched_cols == 4) {
        p.eta = row[2];
        p.inv_a2 = row[3];
        p.k2.eta = make_float2((float)p.eta, (float)p.eta);
        p.k2.inv_a2 = make_float2((float)p.inv_a2, (float)p.inv_a2);
        const float ls = (float)(p.inv_a2 * p.inv_dx2), ne = (float)(-p.eta);
        p.k2.lap_scale = make_float2(ls, ls);
        p.k2.neg_eta = make_float2(ne, ne);
    }
    p.step += s;
}

// Row-blend weight of a 2-D table (same trunc/clamp/unclamped-weight rule
// along T as along phi).
__device__ __forceinline__ void table2d_row(const RealStageParams& p, int& it, double& w) {
    double ft = (p.T - p.T_min) * p.T_dinv;
    double c = ft > 0.0 ? ft : 0.0;
    c = c < double(p.nT - 2) ? c : double(p.nT - 2);
    it = (int)c;
    w = ft - double(it);
}

// Stage the V' row into shared memory as TT (blending the two bracketing T
// rows for a 2-D table).  Called by every thread of the block; ends with a
// barrier.
// Entry q of the row: the 1-D table's value, or the blend of the 2-D table's
// bracketing rows a = it and a + 1 with weight w.
__device__ __forceinline__ double staged_value(const RealStageParams& p, const double* a, double w,
                                               int q) {
    if (p.vkind == TIPT_VP_TABLE) return __ldg(p.table + q);
    const double va = __ldg(a + q), vb = __ldg(a + p.npts + q);
    return va + w * (vb - va);
}

template <typename TT>
__device__ __forceinline__ void stage_table(const RealStageParams& p, TT* s_tab) {
    if (p.vkind == TIPT_VP_TABLE || p.vkind == TIPT_VP_TABLE2D) {
        int it = 0;
        double w = 0.0;
        if (p.vkind == TIPT_VP_TABLE2D) table2d_row(p, it, w);
        const double* a = p.table + (int64_t)it * p.npts;
        for (int q = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
             q < p.npts; q += blockDim.x * blockDim.y * blockDim.z)
            s_tab[q] = (TT)staged_value(p, a, w, q);
    }
    __syncthreads();
}

// The FP32 row as (value, slope) pairs for lerp_pairs_f32: pair q holds the FP32
// value v[q] of stage_table<float> and v[q+1] - v[q] rounded to FP32 (q < npts - 1;
// the lookup never reads the last pair's slope).  Twice the shared memory.
__device__ __forceinline__ void stage_table_pairs(const RealStageParams& p, float2* s_tab2) {
    int it = 0;
    double w = 0.0;
    if (p.vkind == TIPT_VP_TABLE2D) table2d_row(p, it, w);
    const double* a = p.table + (int64_t)it * p.npts;
    for (int q = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); q < p.npts;
         q += blockDim.x * blockDim.y * blockDim.z) {
        const float v = (float)staged_value(p, a, w, q);
        const float d = q + 1 < p.npts ? __fsub_rn((float)staged_value(p, a, w, q + 1), v) : 0.0f;
        s_tab2[q] = make_float2(v, d);
    }
    __syncthreads();
}

// V'(x) in FP64 from the staged row, the global 1-D table, or the polynomial.
// TH = false compiles the thermal branch out (see vprime_v).
template <bool TH = true>
__device__ __forceinline__ double vprime_d(const RealStageParams& p, const double* s_tab, double x) {
    if (p.vkind == TIPT_VP_POLY) return poly_vprime<double>(p.c1, p.c2, p.c3, x);
    if (TH && p.vkind == TIPT_VP_THERMAL) return thermal_vprime_inline(p.th, x);
    const double* t = p.table_in_smem ? s_tab : p.table;
    return lerp_table<double>(t, p.tmin, p.dinv, p.npts - 2, x);
}

// V'(x) in FP32 (F32C storage) for a lane vector: the polynomial, the float
// row staged in shared memory, or (long 1-D tables) the FP64 table in global
// memory.  Lane by lane the same operations as lerp_table<float>.

// FP32 constants of a compensated-FP32 stage, rounded once per launch from the
// FP64 parameters (after the schedule is resolved) and passed to the per-site
// arithmetic, so the loop does no FP64 -> FP32 conversion.
struct F32CConst {
    float h1, h2h, h2l;            // h2 = h2h + h2l
    float inv_dx2, inv_a2, eta, inv_mu2;
    float c1, c2, c3;              // polynomial V'
    float tmin, dinv, last;        // table lookup: (x - tmin) dinv clamped to [0, last]
    float ns;                      // hash noise amplitude
};

// Fills RealStageParams::k2 from the FP64 parameters (host or device).
__host__ __device__ inline void set_f32c_pairs(RealStageParams& p) {
    auto pr = [](float x) { return make_float2(x, x); };
    const float h2h = (float)p.h2;
    p.k2.h1 = pr((float)p.h1);
    p.k2.h2h = pr(h2h);
    p.k2.h2l = pr((float)(p.h2 - (double)h2h));
    p.k2.inv_dx2 = pr((float)p.inv_dx2);
    p.k2.inv_a2 = pr((float)p.inv_a2);
    p.k2.eta = pr((float)p.eta);
    p.k2.inv_mu2 = pr((float)p.inv_mu2);
    p.k2.c1 = pr((float)p.c1);
    p.k2.c2 = pr((float)p.c2);
    p.k2.c3 = pr((float)p.c3);
    p.k2.tmin = pr((float)p.tmin);
    p.k2.dinv = pr((float)p.dinv);
    p.k2.lap_scale = pr((float)(p.inv_a2 * p.inv_dx2));
    p.k2.neg_eta = pr((float)(-p.eta));
    p.k2.neg_imu2 = pr((float)(-p.inv_mu2));
    p.k2.tmd = pr((float)(-p.tmin * p.dinv));
}

// A lane-pair constant as a lane vector.
__device__ __forceinline__ float kv(float2 c, float) { return c.x; }
__device__ __forceinline__ float2 kv(float2 c, float2) { return c; }
template <typename V>
__device__ __forceinline__ V kvec(float2 c) { return kv(c, V{}); }

__device__ __forceinline__ F32CConst f32c_const(const RealStageParams& p) {
    F32CConst k;
    k.h1 = (float)p.h1;
    k.h2h = (float)p.h2;
    k.h2l = (float)(p.h2 - (double)k.h2h);
    k.inv_dx2 = (float)p.inv_dx2;
    k.inv_a2 = (float)p.inv_a2;
    k.eta = (float)p.eta;
    k.inv_mu2 = (float)p.inv_mu2;
    k.c1 = (float)p.c1;
    k.c2 = (float)p.c2;
    k.c3 = (float)p.c3;
    k.tmin = (float)p.tmin;
    k.dinv = (float)p.dinv;
    k.last = (float)(p.npts - 2);
    k.ns = (float)p.ns_eff;
    return k;
}

// TH = false compiles the thermal branch out (kernels launched only for the
// polynomial and table sources keep their register budget).
template <typename V, bool TH = true>
__device__ __forceinline__ V vprime_v(const RealStageParams& p, const F32CConst& kc,
                                      const float* s_tab, V x) {
    constexpr int NL = sizeof(V) / sizeof(float);
    if (p.vkind == TIPT_VP_POLY) {
        const V d = v_fma(v_mul(v_mul(kvec<V>(p.k2.c3), x), x), x, v_mul(kvec<V>(p.k2.c1), x));
        return p.c2 != 0.0 ? v_fma(v_mul(kvec<V>(p.k2.c2), x), x, d) : d;
    }
    if (TH && p.vkind == TIPT_VP_THERMAL) {  // FP64 per lane from the FP32 value
        V r;
#pragma unroll
        for (int l = 0; l < NL; ++l)
            vset(r, l, (float)thermal_vprime_inline(p.th, (double)vlane(x, l)));
        return r;
    }
    if (!p.table_in_smem) {
        V r;
#pragma unroll
        for (int l = 0; l < NL; ++l)
            vset(r, l, (float)lerp_table<double>(p.table, p.tmin, p.dinv, p.npts - 2,
                                                 (double)vlane(x, l)));
        return r;
    }
    // fractional index x dinv - tmin dinv (one rounding; the compensated-FP32 rule)
    return lerp_table_f32<V>(s_tab, v_fma(x, kvec<V>(p.k2.dinv), kvec<V>(p.k2.tmd)), kc.last);
}

// Noise increment for one site (FP64): array value * nfac, or ns_eff * z.
template <typename NT>
__device__ __forceinline__ double site_noise(const RealStageParams& p, uint64_t site) {
    if (p.noise) return __dmul_rn(p.nfac, (double)static_cast<const NT*>(p.noise)[site]);
    if (p.ns_eff == 0.0) return 0.0;
    return __dmul_rn(p.ns_eff, gauss_cos(noise_key(site, p.step, p.mul, p.seed)));
}

// --------------------------------------------------------------- F64 ----
// Stencil order ip, im, jp, jm, kp, km as R:1913-1920.  Every operation is an
// explicit round-to-nearest intrinsic, so each kernel that calls this produces
// the same bits (no compiler-chosen contraction).
__device__ __forceinline__ double sum6_d(const double v[7]) {
    return __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(v[1], v[2]), v[3]), v[4]), v[5]), v[6]);
}
__device__ __forceinline__ double force_d(const RealStageParams& p, double lap, double pv, double dv) {
    // inv_a2*lap - eta*pi - V'/mu^2
    return __dsub_rn(__dsub_rn(__dmul_rn(p.inv_a2, lap), __dmul_rn(p.eta, pv)), __dmul_rn(dv, p.inv_mu2));
}
template <bool TH = true>
__device__ __forceinline__ void update_f64(const RealStageParams& p, const double* s_tab,
                                           const double ph[7], const double pv[7], double noise,
                                           double& phi_new, double& pi_new) {
    const double c = ph[0];
    const double lap = __dmul_rn(__fma_rn(-6.0, c, sum6_d(ph)), p.inv_dx2);
    double pt[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) pt[q] = __fma_rn(p.h1, pv[q], ph[q]);
    const double lap2 = __dmul_rn(__fma_rn(-6.0, pt[0], sum6_d(pt)), p.inv_dx2);
    const double k1 = force_d(p, lap, pv[0], vprime_d<TH>(p, s_tab, c));
    const double pit = __fma_rn(p.h1, k1, pv[0]);
    const double k2 = force_d(p, lap2, pit, vprime_d<TH>(p, s_tab, pt[0]));
    phi_new = __fma_rn(p.h2, pit, c);
    pi_new = __dadd_rn(pv[0], __fma_rn(p.h2, k2, noise));
}

// --------------------------------------------------------------- F32 ----
// The reference's float32 mode (USE_FLOAT32, R:348): float32 neighbour sums,
// FP64 for the rest, float32 stores -- including the stored midpoint state
// phi~, pi~ that pass 2 reads (R:1932-1933).
template <bool TH = true>
__device__ __forceinline__ void update_f32(const RealStageParams& p, const double* s_tab,
                                           const float ph[7], const float pv[7], double noise,
                                           float& phi_new, float& pi_new) {
    const float c = ph[0];
    float s6 = ph[1] + ph[2] + ph[3] + ph[4] + ph[5] + ph[6];
    double lap = ((double)s6 - 6.0 * (double)c) * p.inv_dx2;
    float pt[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) pt[q] = __double2float_rn((double)ph[q] + p.h1 * (double)pv[q]);
    float s6b = pt[1] + pt[2] + pt[3] + pt[4] + pt[5] + pt[6];
    double lap2 = ((double)s6b - 6.0 * (double)pt[0]) * p.inv_dx2;
    double k1 = p.inv_a2 * lap - p.eta * (double)pv[0] - vprime_d<TH>(p, s_tab, (double)c) * p.inv_mu2;
    float pit = __double2float_rn((double)pv[0] + p.h1 * k1);
    double k2 = p.inv_a2 * lap2 - p.eta * (double)pit -
                vprime_d<TH>(p, s_tab, (double)pt[0]) * p.inv_mu2;
    phi_new = __double2float_rn((double)c + p.h2 * (double)pit);
    pi_new = __double2float_rn((double)pv[0] + (p.h2 * k2 + noise));
}

// -------------------------------------------------------------- F32C ----
// Planar {hi, lo} storage (a field is two FP32 planes, value hi + lo), FP32
// arithmetic only, written for lane vectors (one site, or two sites in the
// lanes of the packed FP32x2 instructions).  Forces from hi/lo differences
// (the Laplacian of a smooth field is a difference of nearly equal values:
// hi - hi is exact and the lo parts carry the rest); the state updates
// phi + h2*pi~ and pi + h2*k + kick are float-float (TwoSum), so increments far
// below ulp_fp32(phi) are kept.  `kick` is the noise increment.
//
// Stencil inputs, summed by the caller in the order ip, im, jp, jm, kp, km:
//   dh = sum (hi_n - hi_c),  dl = fma(-6, lo_c, sum lo_n)
template <typename V>
struct F32CIn {
    V dh_phi, dl_phi, dh_pi, dl_pi;  // stencil sums of phi and pi
    V phh, phl, pih, pil;            // centre values
};

template <typename V>
__device__ __forceinline__ V force_v(V inv_a2, V eta, V inv_mu2, V lap, V pv, V dv) {
    return v_sub(v_sub(v_mul(inv_a2, lap), v_mul(eta, pv)), v_mul(dv, inv_mu2));
}

// The same from lapA = inv_a2 lap as two fused multiply-adds (the real field).
template <typename V>
__device__ __forceinline__ V force_fma(V neg_eta, V neg_imu2, V lapA, V pv, V dv) {
    return v_fma(neg_imu2, dv, v_fma(neg_eta, pv, lapA));
}

// The part of the site update that reads only the centre values: the centre
// and midpoint fields and V' at both (marching kernels evaluate it before the
// neighbouring plane arrives).
template <typename V>
struct F32CPre {
    V pvc, v1, v2;  // pi (hi + lo), V'(phi), V'(phi + h1 pi)
};

// The same with the V' source as a functor vp(x) (the batched ensemble's
// per-replica polynomial).
template <typename V, typename VP>
__device__ __forceinline__ F32CPre<V> pre_f32c_vp(const RealStageParams& p, V phh, V phl, V pih,
                                                  V pil, VP vp) {
    const V h1 = kvec<V>(p.k2.h1);
    const V phc = v_add(phh, phl);
    F32CPre<V> r;
    r.pvc = v_add(pih, pil);
    const V pht = v_add(phh, v_fma(h1, r.pvc, phl));
    r.v1 = vp(phc);
    r.v2 = vp(pht);
    return r;
}

template <typename V, bool TH = true>
__device__ __forceinline__ F32CPre<V> pre_f32c(const RealStageParams& p, const F32CConst& kc,
                                               const float* s_tab, V phh, V phl, V pih, V pil) {
    return pre_f32c_vp<V>(p, phh, phl, pih, pil,
                          [&](V x) { return vprime_v<V, TH>(p, kc, s_tab, x); });
}

// Polynomial V'(x) = c1 x + c2 x^2 + c3 x^3 in lane vectors from FP32 pairs: the
// polynomial branch of vprime_v with coefficients given per call.
template <typename V>
__device__ __forceinline__ V poly_vprime_v(float2 c1, float2 c2, float2 c3, bool has_c2, V x) {
    const V d = v_fma(v_mul(v_mul(kvec<V>(c3), x), x), x, v_mul(kvec<V>(c1), x));
    return has_c2 ? v_fma(v_mul(kvec<V>(c2), x), x, d) : d;
}

// The rest of the site update, from the stencil sums, the centre values and the
// pre-part.
template <typename V>
__device__ __forceinline__ void post_f32c(const RealStageParams& p, const F32CIn<V>& x,
                                          const F32CPre<V>& pre, V kick, V& phh, V& phl, V& pih,
                                          V& pil) {
    const V h1 = kvec<V>(p.k2.h1);
    const V h2h = kvec<V>(p.k2.h2h);
    const V h2l = kvec<V>(p.k2.h2l);
    const V lsc = kvec<V>(p.k2.lap_scale);
    const V neg_eta = kvec<V>(p.k2.neg_eta), neg_imu2 = kvec<V>(p.k2.neg_imu2);
    // Laplacians times inv_a2 (inv_a2 inv_dx2 applied once)
    const V lap = v_mul(v_add(x.dh_phi, x.dl_phi), lsc);
    const V lapv = v_mul(v_add(x.dh_pi, x.dl_pi), lsc);
    const V lap2 = v_fma(h1, lapv, lap);  // of phi + h1 pi
    const V pvc = pre.pvc;
    const V k1 = force_fma(neg_eta, neg_imu2, lap, pvc, pre.v1);
    // pi~ = pi + h1 k1 as {t_hi, t_lo}
    V t_hi, t_e;
    two_sum(x.pih, v_mul(h1, k1), t_hi, t_e);
    const V t_lo = v_add(x.pil, t_e);
    const V pit = v_add(t_hi, t_lo);
    const V k2 = force_fma(neg_eta, neg_imu2, lap2, pit, pre.v2);
    // phi + h2 pi~ with the product's rounding error kept
    const V d_hi = v_mul(h2h, t_hi);
    const V d_lo = v_add(v_fma(h2h, t_hi, v_neg(d_hi)), v_fma(h2h, t_lo, v_mul(h2l, t_hi)));
    ff_add(x.phh, x.phl, d_hi, d_lo, phh, phl);
    ff_add1(x.pih, x.pil, v_fma(h2h, k2, kick), pih, pil);
}

template <typename V, bool TH = true>
__device__ __forceinline__ void update_f32c(const RealStageParams& p, const F32CConst& kc,
                                            const float* s_tab, const F32CIn<V>& x, V kick,
                                            V& phh, V& phl, V& pih, V& pil) {
    const F32CPre<V> pre = pre_f32c<V, TH>(p, kc, s_tab, x.phh, x.phl, x.pih, x.pil);
    post_f32c<V>(p, x, pre, kick, phh, phl, pih, pil);
}

// Stencil sums of one planar field for one site from the seven values in
// stencil order (centre, ip, im, jp, jm, kp, km).
__device__ __forceinline__ void stencil_sums(const float hi[7], const float lo[7], float& dh,
                                             float& dl) {
    dh = __fsub_rn(hi[1], hi[0]);
    dl = lo[1];
#pragma unroll
    for (int q = 2; q < 7; ++q) {
        dh = __fadd_rn(dh, __fsub_rn(hi[q], hi[0]));
        dl = __fadd_rn(dl, lo[q]);
    }
    dl = __fmaf_rn(-6.0f, lo[0], dl);
}

// The real-field RK2 stage's order: the i and j terms in sequence, the two k
// terms summed first and added last,
//   dh = (((ip-c) + (im-c)) + (jp-c)) + (jm-c) + ((kp-c) + (km-c)),
//   dl = fma(-6, lo_c, (((ip + im) + jp) + jm) + (kp + km));
// the marching kernel forms the k pair of a site in its own lane (the site's
// k neighbours lie in the neighbouring lanes of its packed pair).
__device__ __forceinline__ void stencil_sums_k(const float hi[7], const float lo[7], float& dh,
                                               float& dl) {
    dh = __fadd_rn(__fsub_rn(hi[1], hi[0]), __fsub_rn(hi[2], hi[0]));
    dh = __fadd_rn(dh, __fsub_rn(hi[3], hi[0]));
    dh = __fadd_rn(dh, __fsub_rn(hi[4], hi[0]));
    dh = __fadd_rn(dh, __fadd_rn(__fsub_rn(hi[5], hi[0]), __fsub_rn(hi[6], hi[0])));
    dl = __fadd_rn(__fadd_rn(__fadd_rn(lo[1], lo[2]), lo[3]), lo[4]);
    dl = __fmaf_rn(-6.0f, lo[0], __fadd_rn(dl, __fadd_rn(lo[5], lo[6])));
}

// Noise increment for one F32C site: array value * nfac, or ns * z (FP32 z).
__device__ __forceinline__ float site_kick_f32c(const RealStageParams& p, const F32CConst& kc,
                                                uint64_t site) {
    if (p.noise) return (float)(p.nfac * static_cast<const double*>(p.noise)[site]);
    if (p.ns_eff == 0.0) return 0.0f;
    return __fmul_rn(kc.ns, gauss_cos_f(noise_key(site, p.step, p.mul, p.seed)));
}
// The same for two consecutive sites (s, s + 1) in the lanes of a float2.
__device__ __forceinline__ float2 site_kick_f32c2(const RealStageParams& p, const F32CConst& kc,
                                                  uint64_t s) {
    if (p.noise) {
        const double* n = static_cast<const double*>(p.noise);
        return make_float2((float)(p.nfac * n[s]), (float)(p.nfac * n[s + 1]));
    }
    if (p.ns_eff == 0.0) return make_float2(0.0f, 0.0f);
    const float2 z = gauss_cos_f2(noise_key(s, p.step, p.mul, p.seed),
                                  noise_key(s + 1, p.step, p.mul, p.seed));
    return v_mul(vs<float2>(kc.ns), z);
}

}  // namespace tipt
