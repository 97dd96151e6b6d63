// Complex-field fused midpoint RK2 stage (C:2067-2215 rk2_step_table) and
// its entry point.  Same single-launch fusion as the real field: the midpoint
// phi~_a = phi_a + h1*pi_a is pointwise, so both reference passes run on the
// 7-point stencil of (phi1, phi2, pi1, pi2).
#include <cstring>

#include "rk2_complex.cuh"
#include "rk2_march.cuh"
#include "tipt_internal.h"

namespace tipt {

template <typename NT>
__device__ __forceinline__ void complex_noise(const ComplexStageParams& p, uint64_t site,
                                              double& n1, double& n2) {
    if (p.noise1) {
        n1 = p.nfac * (double)static_cast<const NT*>(p.noise1)[site];
        n2 = p.nfac * (double)static_cast<const NT*>(p.noise2)[site];
    } else if (p.ns_eff != 0.0) {
        double z1, z2;
        gauss_pair(noise_key(site, p.step, p.mul, p.seed), z1, z2);
        n1 = p.ns_eff * z1;
        n2 = p.ns_eff * z2;
    } else {
        n1 = n2 = 0.0;
    }
}

template <int S, bool TH, bool RG>
__global__ void __launch_bounds__(256) complex_stage_generic(ComplexStageParams p) {
    if constexpr (RG) reset_range_words(p.range_next);
    RangeAcc racc;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using TT = typename std::conditional<S == TIPT_F32C, float, double>::type;
    TT* s_tab = reinterpret_cast<TT*>(smem_raw);
    if (p.table_in_smem) {
        for (int q = threadIdx.x; q < p.npts; q += blockDim.x) s_tab[q] = (TT)__ldg(p.table + q);
        __syncthreads();
    }
    const double* dtab = p.table_in_smem ? reinterpret_cast<const double*>(s_tab) : p.table;
    const int64_t n12 = (int64_t)p.n1 * p.n2;
    const int64_t N = (int64_t)p.n0 * n12;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(s % p.n2);
        const int64_t r = s / p.n2;
        const int j = (int)(r % p.n1);
        const int i = (int)(r / p.n1);
        const int64_t idx[7] = {
            s,
            s + ((i + 1 < p.n0) ? n12 : -(int64_t)(p.n0 - 1) * n12),
            s + ((i > 0) ? -n12 : (int64_t)(p.n0 - 1) * n12),
            s + ((j + 1 < p.n1) ? (int64_t)p.n2 : -(int64_t)(p.n1 - 1) * p.n2),
            s + ((j > 0) ? -(int64_t)p.n2 : (int64_t)(p.n1 - 1) * p.n2),
            s + ((k + 1 < p.n2) ? 1 : -(int64_t)(p.n2 - 1)),
            s + ((k > 0) ? -1 : (int64_t)(p.n2 - 1))};
        if constexpr (S == TIPT_F64) {
            double n1, n2;
            double a[4][7];
#pragma unroll
            for (int f = 0; f < 4; ++f)
#pragma unroll
                for (int q = 0; q < 7; ++q) a[f][q] = __ldg(static_cast<const double*>(p.f[f]) + idx[q]);
            double lap[2], pt[2][7], lapt[2];
#pragma unroll
            for (int f = 0; f < 2; ++f) {
                lap[f] = (a[f][1] + a[f][2] + a[f][3] + a[f][4] + a[f][5] + a[f][6] - 6.0 * a[f][0]) * p.inv_dx2;
#pragma unroll
                for (int q = 0; q < 7; ++q) pt[f][q] = a[f][q] + p.h1 * a[2 + f][q];
                lapt[f] = (pt[f][1] + pt[f][2] + pt[f][3] + pt[f][4] + pt[f][5] + pt[f][6] - 6.0 * pt[f][0]) * p.inv_dx2;
            }
            double d1, d2;
            complex_force<double, TH>(p, dtab, p.tmin, p.dinv, a[0][0], a[1][0], d1, d2);
            double k1a = p.inv_a2 * lap[0] - p.eta * a[2][0] - d1 * p.inv_mu2;
            double k1b = p.inv_a2 * lap[1] - p.eta * a[3][0] - d2 * p.inv_mu2;
            double pta = a[2][0] + p.h1 * k1a, ptb = a[3][0] + p.h1 * k1b;
            complex_force<double, TH>(p, dtab, p.tmin, p.dinv, pt[0][0], pt[1][0], d1, d2);
            double k2a = p.inv_a2 * lapt[0] - p.eta * pta - d1 * p.inv_mu2;
            double k2b = p.inv_a2 * lapt[1] - p.eta * ptb - d2 * p.inv_mu2;
            complex_noise<double>(p, (uint64_t)s, n1, n2);
            const double o0 = a[0][0] + p.h2 * pta, o1 = a[1][0] + p.h2 * ptb;
            static_cast<double*>(p.o[0])[s] = o0;
            static_cast<double*>(p.o[1])[s] = o1;
            static_cast<double*>(p.o[2])[s] = a[2][0] + (p.h2 * k2a + n1);
            static_cast<double*>(p.o[3])[s] = a[3][0] + (p.h2 * k2b + n2);
            if constexpr (RG) fold_rho_f64(racc, o0, o1);
        } else if constexpr (S == TIPT_F32) {
            double n1, n2;
            // float32 storage, FP64 arithmetic after the float32 neighbour sums,
            // float32-rounded midpoint state (as the reference's float32 mode)
            float a[4][7];
#pragma unroll
            for (int f = 0; f < 4; ++f)
#pragma unroll
                for (int q = 0; q < 7; ++q) a[f][q] = __ldg(static_cast<const float*>(p.f[f]) + idx[q]);
            double lap[2], lapt[2];
            float pt[2][7];
#pragma unroll
            for (int f = 0; f < 2; ++f) {
                float s6 = a[f][1] + a[f][2] + a[f][3] + a[f][4] + a[f][5] + a[f][6];
                lap[f] = ((double)s6 - 6.0 * (double)a[f][0]) * p.inv_dx2;
#pragma unroll
                for (int q = 0; q < 7; ++q)
                    pt[f][q] = __double2float_rn((double)a[f][q] + p.h1 * (double)a[2 + f][q]);
                float s6b = pt[f][1] + pt[f][2] + pt[f][3] + pt[f][4] + pt[f][5] + pt[f][6];
                lapt[f] = ((double)s6b - 6.0 * (double)pt[f][0]) * p.inv_dx2;
            }
            double d1, d2;
            complex_force<double, TH>(p, dtab, p.tmin, p.dinv, a[0][0], a[1][0], d1, d2);
            double k1a = p.inv_a2 * lap[0] - p.eta * (double)a[2][0] - d1 * p.inv_mu2;
            double k1b = p.inv_a2 * lap[1] - p.eta * (double)a[3][0] - d2 * p.inv_mu2;
            float pta = __double2float_rn((double)a[2][0] + p.h1 * k1a);
            float ptb = __double2float_rn((double)a[3][0] + p.h1 * k1b);
            complex_force<double, TH>(p, dtab, p.tmin, p.dinv, pt[0][0], pt[1][0], d1, d2);
            double k2a = p.inv_a2 * lapt[0] - p.eta * (double)pta - d1 * p.inv_mu2;
            double k2b = p.inv_a2 * lapt[1] - p.eta * (double)ptb - d2 * p.inv_mu2;
            complex_noise<float>(p, (uint64_t)s, n1, n2);
            const float o0 = __double2float_rn((double)a[0][0] + p.h2 * (double)pta);
            const float o1 = __double2float_rn((double)a[1][0] + p.h2 * (double)ptb);
            static_cast<float*>(p.o[0])[s] = o0;
            static_cast<float*>(p.o[1])[s] = o1;
            if constexpr (RG) racc.fold(rho_f32(o0, o1));
            static_cast<float*>(p.o[2])[s] = __double2float_rn((double)a[2][0] + (p.h2 * k2a + n1));
            static_cast<float*>(p.o[3])[s] = __double2float_rn((double)a[3][0] + (p.h2 * k2b + n2));
        } else {
            // planar {hi, lo} fields; FP32 forces, float-float state updates
            float hi[4][7], lo[4][7];
#pragma unroll
            for (int f = 0; f < 4; ++f)
#pragma unroll
                for (int q = 0; q < 7; ++q) {
                    const float* src = static_cast<const float*>(p.f[f]);
                    hi[f][q] = __ldg(src + idx[q]);
                    lo[f][q] = __ldg(src + N + idx[q]);
                }
            CplxIn<float> in;
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                stencil_sums_k(hi[f], lo[f], in.dh[f], in.dl[f]);
                in.ch[f] = hi[f][0];
                in.cl[f] = lo[f][0];
            }
            const float* ftab = reinterpret_cast<const float*>(s_tab);
            const float h1 = (float)p.h1;
            // The Z_N force of the reference form (C:2152-2158) grows like 1/rho
            // near the origin and amplifies FP32 rounding, so with Z_N active (or a
            // table too large for shared memory) the force is evaluated in FP64 from
            // the full hi + lo values of the centre or the midpoint.
            const bool fp32_force = !(p.zn_active > 0.5 && p.zn_n > 0.5) &&
                                    (p.table_in_smem || p.vkind == TIPT_VP_POLY);
            auto force = [&](float q1, float q2, int which, float& d1, float& d2) {
                if (fp32_force) {
                    complex_force_v<float>(p, ftab, (float)p.tmin, (float)p.dinv, q1, q2, d1, d2);
                } else {
                    double q1d = (double)hi[0][0] + (double)lo[0][0];
                    double q2d = (double)hi[1][0] + (double)lo[1][0];
                    if (which) {
                        q1d = (double)hi[0][0] + ((double)lo[0][0] + (double)h1 * ((double)hi[2][0] + (double)lo[2][0]));
                        q2d = (double)hi[1][0] + ((double)lo[1][0] + (double)h1 * ((double)hi[3][0] + (double)lo[3][0]));
                    }
                    double e1, e2;
                    complex_force<double, TH>(p, p.table, p.tmin, p.dinv, q1d, q2d, e1, e2);
                    d1 = (float)e1;
                    d2 = (float)e2;
                }
            };
            float kick[2] = {0.0f, 0.0f};
            if (p.noise1) {
                kick[0] = (float)(p.nfac * static_cast<const double*>(p.noise1)[s]);
                kick[1] = (float)(p.nfac * static_cast<const double*>(p.noise2)[s]);
            } else {
                complex_kick_f32c(p, (uint64_t)s, kick[0], kick[1]);
            }
            float oh[4], ol[4];
            complex_update_f32c<float>(p, in, kick, force, oh, ol);
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                float* po = static_cast<float*>(p.o[f]);
                po[s] = oh[f];
                po[N + s] = ol[f];
            }
            if constexpr (RG)
                fold_rho_ff(racc, oh[0], ol[0], oh[1], ol[1]);
        }
    }
    if constexpr (RG) racc.flush(p.range);
}

constexpr int64_t kMaxTableSmemC = 96 * 1024;

template <int S>
static int launch_complex_generic(ComplexStageParams p, int64_t smem, cudaStream_t st) {
    auto kern = p.vkind == TIPT_VP_THERMAL
                    ? (p.range ? complex_stage_generic<S, true, true> : complex_stage_generic<S, true, false>)
                    : (p.range ? complex_stage_generic<S, false, true> : complex_stage_generic<S, false, false>);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return fail_cuda(e, "complex_stage smem attribute");
    }
    const int64_t N = (int64_t)p.n0 * p.n1 * p.n2;
    int64_t blocks = (N + 255) / 256;
    const int64_t cap = (int64_t)num_sms() * 8;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, 256, (size_t)smem, st>>>(p);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "complex_stage launch");
}

int launch_complex_stage(int storage, ComplexStageParams p, cudaStream_t st) {
    set_complex_f32(p);
    const bool no_table = p.vkind == TIPT_VP_POLY || p.vkind == TIPT_VP_THERMAL;
    int64_t tb = no_table ? 0 : (int64_t)p.npts * (storage == TIPT_F32C ? 4 : 8);
    p.table_in_smem = (tb > 0 && tb <= kMaxTableSmemC) ? 1 : 0;
    const int64_t smem = p.table_in_smem ? tb : 0;
    if (storage == TIPT_F32C && kernel_policy() != 1) {
        if (complex_march_supported(p)) return launch_complex_march(p, st);
        if (kernel_policy() == 2)
            return fail(TIPT_ERR_UNSUPPORTED, "the complex marching kernel does not take this "
                        "call (Z_N active, noise arrays, table or shape)");
    }
    switch (storage) {
        case TIPT_F64: return launch_complex_generic<TIPT_F64>(p, smem, st);
        case TIPT_F32: return launch_complex_generic<TIPT_F32>(p, smem, st);
        case TIPT_F32C: return launch_complex_generic<TIPT_F32C>(p, smem, st);
    }
    return fail(TIPT_ERR_STORAGE, "unknown storage %d", storage);
}

}  // namespace tipt

using namespace tipt;

// Checks a complex stage call and fills its parameters (one midpoint stage of
// size dt with the pass-2 hash multiplier; callers adjust the half steps).
static int complex_stage_call(int storage, const void* phi1, const void* phi2, const void* pi1,
                              const void* pi2, void* phi1_out, void* phi2_out, void* pi1_out,
                              void* pi2_out, int64_t nx, int64_t ny, int64_t nz,
                              const tipt_step_params* sp, const tipt_vsource* vp,
                              const tipt_complex_terms* ct, const void* noise1,
                              const void* noise2, ComplexStageParams& p) {
    int rc;
    if ((rc = check_state(storage, phi1, phi2, phi1_out, phi2_out, nx, ny, nz)) ||
        (rc = check_state(storage, pi1, pi2, pi1_out, pi2_out, nx, ny, nz)))
        return rc;
    {
        const int64_t bytes = nx * ny * nz * elem_bytes(storage);
        const void* ins[4] = {phi1, phi2, pi1, pi2};
        const void* outs[4] = {phi1_out, phi2_out, pi1_out, pi2_out};
        for (int a = 0; a < 4; ++a) {
            for (int b = 0; b < 4; ++b)
                if (overlap(outs[a], ins[b], bytes))
                    return fail(TIPT_ERR_ARG, "an output array overlaps an input array");
            for (int b = a + 1; b < 4; ++b)
                if (overlap(outs[a], outs[b], bytes))
                    return fail(TIPT_ERR_ARG, "two output arrays overlap");
        }
    }
    if (!sp) return fail(TIPT_ERR_ARG, "step params are NULL");
    if ((rc = check_vsource(vp, "vp"))) return rc;
    if (vp->kind == TIPT_VP_TABLE2D)
        return fail(TIPT_ERR_UNSUPPORTED, "complex field takes a 1-D V'(rho) table");
    if ((noise1 == nullptr) != (noise2 == nullptr))
        return fail(TIPT_ERR_ARG, "noise1 and noise2 must both be given or both be NULL");
    if (noise1 && ((rc = check_ptr(noise1, storage == TIPT_F32 ? 4 : 8, "noise1")) ||
                   (rc = check_ptr(noise2, storage == TIPT_F32 ? 4 : 8, "noise2"))))
        return rc;
    memset(&p, 0, sizeof(p));
    p.f[0] = phi1;
    p.f[1] = phi2;
    p.f[2] = pi1;
    p.f[3] = pi2;
    p.o[0] = phi1_out;
    p.o[1] = phi2_out;
    p.o[2] = pi1_out;
    p.o[3] = pi2_out;
    p.n0 = (int)nx;
    p.n1 = (int)ny;
    p.n2 = (int)nz;
    p.h1 = 0.5 * sp->dt;
    p.h2 = sp->dt;
    p.inv_dx2 = 1.0 / (sp->dx * sp->dx);
    p.eta = sp->eta_eff;
    p.inv_mu2 = 1.0 / (sp->mu * sp->mu);
    p.inv_a2 = sp->inv_a2;
    p.noise1 = noise1;
    p.noise2 = noise2;
    p.ns_eff = sp->noise_scale;
    p.nfac = 1.0;
    p.step = sp->noise_step;
    p.mul = kPass2Mul;
    p.seed = sp->noise_seed;
    if (ct) {
        p.zn_n = ct->zn_n;
        p.zn_dv = ct->zn_dv;
        p.zn_active = ct->zn_active;
        p.eps4 = ct->eps4;
    }
    p.vkind = vp->kind;
    p.npts = vp->npts;
    p.table = vp->table;
    p.tmin = vp->tmin;
    p.dinv = vp->dinv;
    p.c1 = vp->c1;
    p.c2 = vp->c2;
    p.c3 = vp->c3;
    if (vp->kind == TIPT_VP_THERMAL) p.th = thermal_site(*vp->thermal, vp->T);
    return TIPT_OK;
}


extern "C" int tipt_complex_rk2_step_table(int storage, const void* phi1, const void* phi2,
                                           const void* pi1, const void* pi2, void* phi1_out,
                                           void* phi2_out, void* pi1_out, void* pi2_out, int64_t nx,
                                           int64_t ny, int64_t nz, const tipt_step_params* sp,
                                           const tipt_vsource* vp,
                                           const tipt_complex_terms* ct, const void* noise1,
                                           const void* noise2, void* stream) {
    ComplexStageParams p;
    int rc = complex_stage_call(storage, phi1, phi2, pi1, pi2, phi1_out, phi2_out, pi1_out,
                                pi2_out, nx, ny, nz, sp, vp, ct, noise1, noise2, p);
    if (rc) return rc;
    return launch_complex_stage(storage, p, (cudaStream_t)stream);
}

extern "C" int tipt_complex_rk2_step_table_range(int storage, const void* phi1, const void* phi2,
                                                 const void* pi1, const void* pi2, void* phi1_out,
                                                 void* phi2_out, void* pi1_out, void* pi2_out,
                                                 int64_t nx, int64_t ny, int64_t nz,
                                                 const tipt_step_params* sp,
                                                 const tipt_vsource* vp,
                                                 const tipt_complex_terms* ct, const void* noise1,
                                                 const void* noise2, uint32_t* range,
                                                 uint32_t* range_next, void* stream) {
    ComplexStageParams p;
    int rc = complex_stage_call(storage, phi1, phi2, pi1, pi2, phi1_out, phi2_out, pi1_out,
                                pi2_out, nx, ny, nz, sp, vp, ct, noise1, noise2, p);
    if (rc) return rc;
    if ((rc = check_ptr(range, 4, "range")) || (rc = check_ptr(range_next, 4, "range_next")))
        return rc;
    if (overlap(range, range_next, 12)) return fail(TIPT_ERR_ARG, "range and range_next overlap");
    p.range = reinterpret_cast<unsigned int*>(range);
    p.range_next = reinterpret_cast<unsigned int*>(range_next);
    return launch_complex_stage(storage, p, (cudaStream_t)stream);
}

extern "C" int tipt_complex_rk2_fused_table(int storage, const void* phi1, const void* phi2,
                                            const void* pi1, const void* pi2, void* phi1_out,
                                            void* phi2_out, void* pi1_out, void* pi2_out,
                                            void* mid1, void* mid2, void* mid3, void* mid4,
                                            int64_t nx, int64_t ny, int64_t nz,
                                            const tipt_step_params* sp,
                                            const tipt_vsource* vp_T, const tipt_vsource* vp_Tm,
                                            const tipt_complex_terms* ct, const void* noise1,
                                            const void* noise2, void* stream) {
    ComplexStageParams a, b;
    int rc = complex_stage_call(storage, phi1, phi2, pi1, pi2, mid1, mid2, mid3, mid4, nx, ny, nz,
                                sp, vp_T, ct, noise1, noise2, a);
    if (rc) return rc;
    rc = complex_stage_call(storage, mid1, mid2, mid3, mid4, phi1_out, phi2_out, pi1_out, pi2_out,
                            nx, ny, nz, sp, vp_Tm, ct, noise1, noise2, b);
    if (rc) return rc;
    // first half at T (C:1829-1946), pass-2 multiplier; second at T_mid
    // (C:1948-2064), pass-4 multiplier; 0.5 noise (array or hash) in each
    for (ComplexStageParams* q : {&a, &b}) {
        q->h1 = q->h2 = 0.5 * sp->dt;
        q->nfac = 0.5;
        q->ns_eff = 0.5 * sp->noise_scale;
    }
    b.mul = kPass4Mul;
    if ((rc = launch_complex_stage(storage, a, (cudaStream_t)stream))) return rc;
    return launch_complex_stage(storage, b, (cudaStream_t)stream);
}
