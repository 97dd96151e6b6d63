// Alternative integrators of the reference: BAOAB (R:1974-2108, C:2223-2414)
// and overdamped Euler-Maruyama (R:2115-2193, C:2422-2528), real and complex
// field, with counter-based hash noise.
//
// The reference kernels update the field in place inside a parallel loop
// (a site may read neighbours already advanced in the same sweep) and draw
// numpy Mersenne-Twister normals, so a run is not reproducible even against
// itself.  Here every sub-step reads the previous sub-step's state only
// (ping-pong outputs), which is the splitting the reference's docstrings
// state:
//   overdamped:  phi' = phi + dt/eta F(phi) + ns z
//   BAOAB:       pass 1  pi' = pi + h F(phi); phi' = phi + h pi';
//                        pi'' = c1 pi' + c2 z; phi'' = phi' + h pi''
//                pass 2  pi''' = pi'' + h F(phi'')
// with h = dt/2, c1 = exp(-gamma dt), c2 = sqrt(1 - c1^2) ns,
// F = inv_a2 lap(phi) - V'(phi) inv_mu2 (complex: V'(rho) projected, Z_N).
// Noise: z = Box-Muller of the hash of (site, step) at the pass-2 multiplier;
// the complex field takes the cosine and sine branches of one pair.
// Storages: F64 (FP64), F32 (the reference's float32 mode: FP32 neighbour
// sums, FP64 arithmetic, FP32 stores after each sub-step), F32C (FP32 forces,
// float-float state updates).
#include <cstring>

#include "integrators.cuh"
#include "rk2_march.cuh"
#include "tipt_internal.h"

namespace tipt {

// FP64 Laplacian in the reference order (ip, im, jp, jm, kp, km, then - 6 c).
__device__ __forceinline__ double lap_d(const double q[7], double inv_dx2) {
    double s = __dadd_rn(q[1], q[2]);
#pragma unroll
    for (int n = 3; n < 7; ++n) s = __dadd_rn(s, q[n]);
    return __dmul_rn(__dsub_rn(s, __dmul_rn(6.0, q[0])), inv_dx2);
}
// float32 storage: FP32 neighbour sum, then FP64 (the reference's float32 mode).
__device__ __forceinline__ double lap_f(const float q[7], double inv_dx2) {
    float s = __fadd_rn(q[1], q[2]);
#pragma unroll
    for (int n = 3; n < 7; ++n) s = __fadd_rn(s, q[n]);
    return __dmul_rn(__dsub_rn((double)s, __dmul_rn(6.0, (double)q[0])), inv_dx2);
}

__device__ __forceinline__ double vprime_alt_d(const ComplexStageParams& v, const double* tab,
                                               double x) {
    if (v.vkind == TIPT_VP_POLY) return poly_vprime<double>(v.c1, v.c2, v.c3, x);
    return lerp_table<double>(tab, v.tmin, v.dinv, v.npts - 2, x);
}
__device__ __forceinline__ double force_d(const AltParams& p, double lap, double dv) {
    return __dsub_rn(__dmul_rn(p.inv_a2, lap), __dmul_rn(dv, p.inv_mu2));
}

template <typename TT>
__device__ __forceinline__ const TT* stage_alt_table(const AltParams& p, TT* s_tab) {
    if (p.v.table_in_smem) {
        for (int q = threadIdx.x; q < p.v.npts; q += blockDim.x) s_tab[q] = (TT)__ldg(p.v.table + q);
        __syncthreads();
    }
    return s_tab;
}

// ----------------------------------------------------------------- real ----
template <int S, int MODE>
__global__ void __launch_bounds__(256) alt_real_kernel(AltParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using TT = typename std::conditional<S == TIPT_F32C, float, double>::type;
    const TT* s_tab = stage_alt_table<TT>(p, reinterpret_cast<TT*>(smem_raw));
    const double* dtab = p.v.table_in_smem ? reinterpret_cast<const double*>(s_tab) : p.v.table;
    const int64_t n12 = (int64_t)p.n1 * p.n2;
    const int64_t N = (int64_t)p.n0 * n12;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(s % p.n2);
        const int64_t r = s / p.n2;
        const int j = (int)(r % p.n1);
        const int i = (int)(r / p.n1);
        const int64_t idx[7] = {
            s, s + ((i + 1 < p.n0) ? n12 : -(int64_t)(p.n0 - 1) * n12),
            s + ((i > 0) ? -n12 : (int64_t)(p.n0 - 1) * n12),
            s + ((j + 1 < p.n1) ? (int64_t)p.n2 : -(int64_t)(p.n1 - 1) * p.n2),
            s + ((j > 0) ? -(int64_t)p.n2 : (int64_t)(p.n1 - 1) * p.n2),
            s + ((k + 1 < p.n2) ? 1 : -(int64_t)(p.n2 - 1)), s + ((k > 0) ? -1 : (int64_t)(p.n2 - 1))};
        const bool noisy = (MODE == kOD && p.ns != 0.0) || (MODE == kBA1 && p.c2 != 0.0);
        const uint64_t key = noise_key((uint64_t)s, p.step, kPass2Mul, p.seed);
        if constexpr (S == TIPT_F64 || S == TIPT_F32) {
            using E = typename std::conditional<S == TIPT_F64, double, float>::type;
            const E* phi = static_cast<const E*>(p.f[0]);
            E q[7];
#pragma unroll
            for (int n = 0; n < 7; ++n) q[n] = __ldg(phi + idx[n]);
            double lap;
            if constexpr (S == TIPT_F64) lap = lap_d(q, p.inv_dx2);
            else lap = lap_f(q, p.inv_dx2);
            const double ph = (double)q[0];
            const double F = force_d(p, lap, vprime_alt_d(p.v, dtab, ph));
            const double z = noisy ? gauss_cos(key) : 0.0;
            if constexpr (MODE == kOD) {
                static_cast<E*>(p.o[0])[s] =
                    (E)__dadd_rn(__dadd_rn(ph, __dmul_rn(p.dto, F)), __dmul_rn(p.ns, z));
            } else {
                double pv = (double)static_cast<const E*>(p.f[1])[s];
                if constexpr (MODE == kBA1) {
                    pv = (double)(E)__dadd_rn(pv, __dmul_rn(p.h, F));
                    const double pa = (double)(E)__dadd_rn(ph, __dmul_rn(p.h, pv));
                    const double po = (double)(E)__dadd_rn(__dmul_rn(p.c1, pv), __dmul_rn(p.c2, z));
                    static_cast<E*>(p.o[0])[s] = (E)__dadd_rn(pa, __dmul_rn(p.h, po));
                    static_cast<E*>(p.o[1])[s] = (E)po;
                } else {
                    static_cast<E*>(p.o[1])[s] = (E)__dadd_rn(pv, __dmul_rn(p.h, F));
                }
            }
        } else {
            const float* phi = static_cast<const float*>(p.f[0]);
            float hh[7], hl[7];
#pragma unroll
            for (int n = 0; n < 7; ++n) {
                hh[n] = __ldg(phi + idx[n]);
                hl[n] = __ldg(phi + N + idx[n]);
            }
            float dh, dl;
            stencil_sums(hh, hl, dh, dl);
            const float vp = vprime_alt_f(p.v, s_tab, __fadd_rn(hh[0], hl[0]));
            const float z = noisy ? gauss_cos_f(key) : 0.0f;
            float* out0 = static_cast<float*>(p.o[0]);
            float* out1 = static_cast<float*>(p.o[1]);
            float vh = 0.0f, vl = 0.0f, ah, al, bh, bl;
            if constexpr (MODE != kOD) {
                const float* pif = static_cast<const float*>(p.f[1]);
                vh = pif[s];
                vl = pif[N + s];
            }
            alt_real_site_f32c<MODE>(p, hh[0], hl[0], dh, dl, vp, z, vh, vl, ah, al, bh, bl);
            if constexpr (MODE != kBA2) {
                out0[s] = ah;
                out0[N + s] = al;
            }
            if constexpr (MODE != kOD) {
                out1[s] = bh;
                out1[N + s] = bl;
            }
        }
    }
}

// -------------------------------------------------------------- complex ----
template <int S, int MODE>
__global__ void __launch_bounds__(256) alt_complex_kernel(AltParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using TT = typename std::conditional<S == TIPT_F32C, float, double>::type;
    const TT* s_tab = stage_alt_table<TT>(p, reinterpret_cast<TT*>(smem_raw));
    const double* dtab = p.v.table_in_smem ? reinterpret_cast<const double*>(s_tab) : p.v.table;
    const bool zn = p.v.zn_active > 0.5 && p.v.zn_n > 0.5;
    const int64_t n12 = (int64_t)p.n1 * p.n2;
    const int64_t N = (int64_t)p.n0 * n12;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(s % p.n2);
        const int64_t r = s / p.n2;
        const int j = (int)(r % p.n1);
        const int i = (int)(r / p.n1);
        const int64_t idx[7] = {
            s, s + ((i + 1 < p.n0) ? n12 : -(int64_t)(p.n0 - 1) * n12),
            s + ((i > 0) ? -n12 : (int64_t)(p.n0 - 1) * n12),
            s + ((j + 1 < p.n1) ? (int64_t)p.n2 : -(int64_t)(p.n1 - 1) * p.n2),
            s + ((j > 0) ? -(int64_t)p.n2 : (int64_t)(p.n1 - 1) * p.n2),
            s + ((k + 1 < p.n2) ? 1 : -(int64_t)(p.n2 - 1)), s + ((k > 0) ? -1 : (int64_t)(p.n2 - 1))};
        const bool noisy = (MODE == kOD && p.ns != 0.0) || (MODE == kBA1 && p.c2 != 0.0);
        const uint64_t key = noise_key((uint64_t)s, p.step, kPass2Mul, p.seed);
        if constexpr (S == TIPT_F64 || S == TIPT_F32) {
            using E = typename std::conditional<S == TIPT_F64, double, float>::type;
            double lap[2], c[2];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const E* ph = static_cast<const E*>(p.f[a]);
                E q[7];
#pragma unroll
                for (int n = 0; n < 7; ++n) q[n] = __ldg(ph + idx[n]);
                if constexpr (S == TIPT_F64) lap[a] = lap_d(q, p.inv_dx2);
                else lap[a] = lap_f(q, p.inv_dx2);
                c[a] = (double)q[0];
            }
            double d1, d2;
            complex_force<double, false>(p.v, dtab, p.v.tmin, p.v.dinv, c[0], c[1], d1, d2);
            const double F[2] = {force_d(p, lap[0], d1), force_d(p, lap[1], d2)};
            double z[2] = {0.0, 0.0};
            if (noisy) gauss_pair(key, z[0], z[1]);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                if constexpr (MODE == kOD) {
                    static_cast<E*>(p.o[a])[s] = (E)__dadd_rn(__dadd_rn(c[a], __dmul_rn(p.dto, F[a])),
                                                             __dmul_rn(p.ns, z[a]));
                } else {
                    double pv = (double)static_cast<const E*>(p.f[2 + a])[s];
                    if constexpr (MODE == kBA1) {
                        pv = (double)(E)__dadd_rn(pv, __dmul_rn(p.h, F[a]));
                        const double pa = (double)(E)__dadd_rn(c[a], __dmul_rn(p.h, pv));
                        const double po =
                            (double)(E)__dadd_rn(__dmul_rn(p.c1, pv), __dmul_rn(p.c2, z[a]));
                        static_cast<E*>(p.o[a])[s] = (E)__dadd_rn(pa, __dmul_rn(p.h, po));
                        static_cast<E*>(p.o[2 + a])[s] = (E)po;
                    } else {
                        static_cast<E*>(p.o[2 + a])[s] = (E)__dadd_rn(pv, __dmul_rn(p.h, F[a]));
                    }
                }
            }
        } else {
            float ch[2], cl[2], lap[2];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const float* ph = static_cast<const float*>(p.f[a]);
                float hh[7], hl[7];
#pragma unroll
                for (int n = 0; n < 7; ++n) {
                    hh[n] = __ldg(ph + idx[n]);
                    hl[n] = __ldg(ph + N + idx[n]);
                }
                float dh, dl;
                stencil_sums(hh, hl, dh, dl);
                lap[a] = __fmul_rn(__fadd_rn(dh, dl), (float)p.inv_dx2);
                ch[a] = hh[0];
                cl[a] = hl[0];
            }
            float d1, d2;
            if (!zn && (p.v.table_in_smem || p.v.vkind == TIPT_VP_POLY)) {
                complex_force_v<float>(p.v, s_tab, (float)p.v.tmin, (float)p.v.dinv,
                                       __fadd_rn(ch[0], cl[0]), __fadd_rn(ch[1], cl[1]), d1, d2);
            } else {
                double e1, e2;
                complex_force<double, false>(p.v, p.v.table, p.v.tmin, p.v.dinv,
                                      (double)ch[0] + (double)cl[0], (double)ch[1] + (double)cl[1],
                                      e1, e2);
                d1 = (float)e1;
                d2 = (float)e2;
            }
            const float dv[2] = {d1, d2};
            float z[2] = {0.0f, 0.0f};
            if (noisy) gauss_pair_f(key, z[0], z[1]);
            const float h = (float)p.h, hlo = (float)(p.h - (double)h);
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const float F = __fsub_rn(__fmul_rn((float)p.inv_a2, lap[a]),
                                          __fmul_rn(dv[a], (float)p.inv_mu2));
                float* out = static_cast<float*>(p.o[a]);
                float* outp = static_cast<float*>(p.o[2 + a]);
                if constexpr (MODE == kOD) {
                    float x, y;
                    ff_add(ch[a], cl[a], __fmaf_rn((float)p.dto, F, __fmul_rn((float)p.ns, z[a])),
                           0.0f, x, y);
                    out[s] = x;
                    out[N + s] = y;
                } else {
                    const float* pif = static_cast<const float*>(p.f[2 + a]);
                    float vh = pif[s], vl = pif[N + s];
                    if constexpr (MODE == kBA1) {
                        ff_add(vh, vl, __fmul_rn(h, F), 0.0f, vh, vl);
                        float ah, al;
                        ff_axpy(ch[a], cl[a], h, hlo, vh, vl, ah, al);
                        const float c1h = (float)p.c1, c1l = (float)(p.c1 - (double)c1h);
                        const float ph_ = __fmul_rn(c1h, vh);
                        const float pl_ = __fadd_rn(__fmaf_rn(c1h, vh, -ph_),
                                                    __fmaf_rn(c1h, vl, __fmul_rn(c1l, vh)));
                        float oh, ol;
                        ff_add(ph_, pl_, __fmul_rn((float)p.c2, z[a]), 0.0f, oh, ol);
                        float fh, fl;
                        ff_axpy(ah, al, h, hlo, oh, ol, fh, fl);
                        out[s] = fh;
                        out[N + s] = fl;
                        outp[s] = oh;
                        outp[N + s] = ol;
                    } else {
                        float oh, ol;
                        ff_add(vh, vl, __fmul_rn(h, F), 0.0f, oh, ol);
                        outp[s] = oh;
                        outp[N + s] = ol;
                    }
                }
            }
        }
    }
}

// ------------------------------------------------------------------ host ----
constexpr int64_t kMaxAltTableSmem = 96 * 1024;

template <int S, int MODE, bool CPLX>
static int launch_alt_k(const AltParams& p, cudaStream_t st) {
    auto kern = CPLX ? alt_complex_kernel<S, MODE> : alt_real_kernel<S, MODE>;
    const int64_t smem = p.v.table_in_smem ? (int64_t)p.v.npts * (S == TIPT_F32C ? 4 : 8) : 0;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return fail_cuda(e, "integrator smem attribute");
    }
    const int64_t N = (int64_t)p.n0 * p.n1 * p.n2;
    int64_t blocks = (N + 255) / 256;
    const int64_t cap = (int64_t)num_sms() * 8;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, 256, (size_t)smem, st>>>(p);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "integrator launch");
}

template <int MODE, bool CPLX>
static int launch_alt(int storage, const AltParams& p, cudaStream_t st) {
    // compensated FP32 on the marching ring where the shape allows (bitwise the
    // generic kernel's results; kernel_policy 1 forces the generic one)
    if (storage == TIPT_F32C && kernel_policy() != 1 && alt_march_supported(p, CPLX))
        return launch_alt_march(MODE, CPLX, p, st);
    switch (storage) {
        case TIPT_F64: return launch_alt_k<TIPT_F64, MODE, CPLX>(p, st);
        case TIPT_F32: return launch_alt_k<TIPT_F32, MODE, CPLX>(p, st);
        case TIPT_F32C: return launch_alt_k<TIPT_F32C, MODE, CPLX>(p, st);
    }
    return fail(TIPT_ERR_STORAGE, "unknown storage %d", storage);
}

// Shared argument checks; fills the scalars and the V' source of `p`.
static int alt_setup(int storage, const void* const* in, int n_in, void* const* out, int n_out,
                     int64_t nx, int64_t ny, int64_t nz, const tipt_step_params* sp,
                     const tipt_vsource* vp, const tipt_complex_terms* ct, AltParams& p) {
    int rc;
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz))) return rc;
    const int ea = elem_align(storage);
    for (int a = 0; a < n_in; ++a)
        if ((rc = check_ptr(in[a], ea, "input field"))) return rc;
    for (int a = 0; a < n_out; ++a)
        if ((rc = check_ptr(out[a], ea, "output field"))) return rc;
    const int64_t bytes = nx * ny * nz * elem_bytes(storage);
    for (int a = 0; a < n_out; ++a) {
        for (int b = 0; b < n_in; ++b)
            if (overlap(out[a], in[b], bytes))
                return fail(TIPT_ERR_ARG, "an output field overlaps an input field (the stencil "
                            "reads neighbours: ping-pong the buffers)");
        for (int b = a + 1; b < n_out; ++b)
            if (overlap(out[a], out[b], bytes)) return fail(TIPT_ERR_ARG, "two outputs overlap");
    }
    if (!sp) return fail(TIPT_ERR_ARG, "step params are NULL");
    if ((rc = check_vsource(vp, "vp"))) return rc;
    if (vp->kind == TIPT_VP_TABLE2D || vp->kind == TIPT_VP_THERMAL)
        return fail(TIPT_ERR_UNSUPPORTED, "these integrators take a 1-D V' table or a polynomial");
    if (!(sp->dt > 0.0) || !(sp->eta_eff > 0.0))
        return fail(TIPT_ERR_ARG, "dt and eta_eff (gamma) must be > 0");
    memset(&p, 0, sizeof(p));
    p.n0 = (int)nx;
    p.n1 = (int)ny;
    p.n2 = (int)nz;
    p.h = 0.5 * sp->dt;
    p.dto = sp->dt / sp->eta_eff;
    p.inv_dx2 = 1.0 / (sp->dx * sp->dx);
    p.inv_mu2 = 1.0 / (sp->mu * sp->mu);
    p.inv_a2 = sp->inv_a2;
    p.c1 = exp(-sp->eta_eff * sp->dt);
    p.c2 = sqrt(1.0 - p.c1 * p.c1) * sp->noise_scale;
    p.ns = sp->noise_scale;
    p.step = sp->noise_step;
    p.seed = sp->noise_seed;
    p.v.vkind = vp->kind;
    p.v.npts = vp->npts;
    p.v.table = vp->table;
    p.v.tmin = vp->tmin;
    p.v.dinv = vp->dinv;
    p.v.c1 = vp->c1;
    p.v.c2 = vp->c2;
    p.v.c3 = vp->c3;
    const int64_t tb = vp->kind == TIPT_VP_POLY ? 0 : (int64_t)vp->npts * (storage == TIPT_F32C ? 4 : 8);
    p.v.table_in_smem = (tb > 0 && tb <= kMaxAltTableSmem) ? 1 : 0;
    if (ct) {
        p.v.zn_n = ct->zn_n;
        p.v.zn_dv = ct->zn_dv;
        p.v.zn_active = ct->zn_active;
        p.v.eps4 = ct->eps4;
    }
    return TIPT_OK;
}

}  // namespace tipt

using namespace tipt;

extern "C" int tipt_overdamped_step_table(int storage, const void* phi, void* phi_out, int64_t nx,
                                          int64_t ny, int64_t nz, const tipt_step_params* sp,
                                          const tipt_vsource* vp, void* stream) {
    AltParams p;
    const void* in[1] = {phi};
    void* out[1] = {phi_out};
    int rc = alt_setup(storage, in, 1, out, 1, nx, ny, nz, sp, vp, nullptr, p);
    if (rc) return rc;
    p.f[0] = phi;
    p.o[0] = phi_out;
    return launch_alt<kOD, false>(storage, p, (cudaStream_t)stream);
}

extern "C" int tipt_baoab_step_table(int storage, const void* phi, const void* pi, void* phi_out,
                                     void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                                     const tipt_step_params* sp, const tipt_vsource* vp,
                                     void* stream) {
    AltParams p;
    const void* in[2] = {phi, pi};
    void* out[2] = {phi_out, pi_out};
    int rc = alt_setup(storage, in, 2, out, 2, nx, ny, nz, sp, vp, nullptr, p);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    p.f[0] = phi;
    p.f[1] = pi;
    p.o[0] = phi_out;
    p.o[1] = pi_out;
    if ((rc = launch_alt<kBA1, false>(storage, p, st))) return rc;
    // pass 2 reads phi'' (stencil) and pi'' at its own site only: pi updated in place
    p.f[0] = phi_out;
    p.f[1] = pi_out;
    p.o[0] = nullptr;
    p.o[1] = pi_out;
    return launch_alt<kBA2, false>(storage, p, st);
}

extern "C" int tipt_complex_overdamped_step_table(int storage, const void* phi1, const void* phi2,
                                                  void* phi1_out, void* phi2_out, int64_t nx,
                                                  int64_t ny, int64_t nz,
                                                  const tipt_step_params* sp,
                                                  const tipt_vsource* vp,
                                                  const tipt_complex_terms* ct, void* stream) {
    AltParams p;
    const void* in[2] = {phi1, phi2};
    void* out[2] = {phi1_out, phi2_out};
    int rc = alt_setup(storage, in, 2, out, 2, nx, ny, nz, sp, vp, ct, p);
    if (rc) return rc;
    p.f[0] = phi1;
    p.f[1] = phi2;
    p.o[0] = phi1_out;
    p.o[1] = phi2_out;
    return launch_alt<kOD, true>(storage, p, (cudaStream_t)stream);
}

extern "C" int tipt_complex_baoab_step_table(int storage, const void* phi1, const void* phi2,
                                             const void* pi1, const void* pi2, void* phi1_out,
                                             void* phi2_out, void* pi1_out, void* pi2_out,
                                             int64_t nx, int64_t ny, int64_t nz,
                                             const tipt_step_params* sp, const tipt_vsource* vp,
                                             const tipt_complex_terms* ct, void* stream) {
    AltParams p;
    const void* in[4] = {phi1, phi2, pi1, pi2};
    void* out[4] = {phi1_out, phi2_out, pi1_out, pi2_out};
    int rc = alt_setup(storage, in, 4, out, 4, nx, ny, nz, sp, vp, ct, p);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    for (int a = 0; a < 4; ++a) {
        p.f[a] = in[a];
        p.o[a] = out[a];
    }
    if ((rc = launch_alt<kBA1, true>(storage, p, st))) return rc;
    for (int a = 0; a < 4; ++a) p.f[a] = out[a];
    p.o[0] = p.o[1] = nullptr;
    return launch_alt<kBA2, true>(storage, p, st);
}
