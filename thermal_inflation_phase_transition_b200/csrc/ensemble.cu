// Batched ensemble of independent real-field replicas with uneven lattice
// sizes, seeds and potentials, advanced by one persistent launch per step.
//
// The reference runs one replica per CLI invocation (one numba call per
// step).  Here every replica's state is a slice of one packed buffer (planar
// for the compensated storage: hi plane of all replicas, then the lo plane);
// a work-list of chunks (replica, site range) covers the active replicas and
// persistent CTAs walk it, so a step of 1792 small replicas is one launch
// instead of 1792.  Each site runs the same midpoint arithmetic as the
// single-lattice kernels, with the replica's own extents, noise seed and
// amplitude, and polynomial V'(phi) = c1 phi + c2 phi^2 + c3 phi^3 (the
// potential family's derivative: c1 = 2D(T^2-T0^2), c2 = -3ET, c3 = lam).
// Results are bitwise those of stepping the replica alone with the generic
// kernel.
//
// tipt_ensemble_observe reduces, per replica and in a fixed order, the
// fraction of sites with phi > thr; the first time it exceeds the stop
// fraction the step is recorded as the replica's first-passage step, and once
// it exceeds the retire fraction (>= the stop fraction) the replica is retired
// (its chunks are skipped from then on).
#include <cstring>

#include "rk2_march.cuh"
#include "rk2_real.cuh"
#include "tipt_internal.h"

namespace tipt {

struct EnsParams {
    const void* phi;
    const void* pi;
    void* phi_out;
    void* pi_out;
    int64_t n_total;
    const tipt_replica* reps;
    const tipt_chunk* chunks;
    int n_chunks;
    const int32_t* active;
    double h1, h2, inv_dx2, eta, inv_mu2, inv_a2;
    uint64_t step;                       // hash step = step (+ *ctr + offset)
    const unsigned long long* ctr;       // device step counter or nullptr
    long long offset;
};

// x / d for x < 2^32 / d by a multiply-high with m = ceil(2^32 / d) (exact:
// x m / 2^32 = x/d + x e / (d 2^32) with e = m d - 2^32 < d); m = 0 means d = 1.
__device__ __forceinline__ uint32_t fdiv(uint32_t x, uint32_t m) { return m ? __umulhi(x, m) : x; }

template <int S>
__global__ void __launch_bounds__(256) ensemble_stage_kernel(EnsParams e) {
    const uint64_t step = e.step + (e.ctr ? *e.ctr + (unsigned long long)e.offset : 0ull);
    for (int c = blockIdx.x; c < e.n_chunks; c += gridDim.x) {
        const tipt_chunk ch = e.chunks[c];
        if (!e.active[ch.replica]) continue;
        const tipt_replica rp = e.reps[ch.replica];
        // the replica as a single lattice with a polynomial V' and hash noise
        RealStageParams p;
        memset(&p, 0, sizeof(p));
        p.n0 = rp.n0;
        p.n1 = rp.n1;
        p.n2 = rp.n2;
        p.h1 = e.h1;
        p.h2 = e.h2;
        p.inv_dx2 = e.inv_dx2;
        p.eta = e.eta;
        p.inv_mu2 = e.inv_mu2;
        p.inv_a2 = e.inv_a2;
        p.ns_eff = rp.noise_scale;
        p.nfac = 1.0;
        p.step = step;
        p.mul = kPass2Mul;
        p.seed = rp.seed;
        p.vkind = TIPT_VP_POLY;
        p.c1 = rp.c1;
        p.c2 = rp.c2;
        p.c3 = rp.c3;
        const uint32_t n12 = (uint32_t)rp.n1 * (uint32_t)rp.n2;
        set_f32c_pairs(p);
        const F32CConst kc = f32c_const(p);
        if constexpr (S == TIPT_F32C) {
            // Site pairs (s, s + 1) with s even share i and j when n2 is even: one
            // 8-byte load per field plane and neighbour, the stencil sums and the
            // update in the lanes of the packed FP32x2 instructions (bitwise the
            // one-site arithmetic, as in the marching kernel).
            if ((rp.n2 & 1) == 0 && ((ch.begin | ch.count | rp.offset) & 1) == 0) {
                const float* phi = static_cast<const float*>(e.phi);
                const float* pi = static_cast<const float*>(e.pi);
                float* po = static_cast<float*>(e.phi_out);
                float* vo = static_cast<float*>(e.pi_out);
                const int64_t N = e.n_total;
                for (int t = threadIdx.x; 2 * t < ch.count; t += blockDim.x) {
                    const uint32_t s = (uint32_t)(ch.begin + 2 * t);
                    const uint32_t q = fdiv(s, rp.m2);
                    const uint32_t k = s - q * (uint32_t)rp.n2;
                    const uint32_t i = fdiv(q, rp.m1);
                    const uint32_t j = q - i * (uint32_t)rp.n1;
                    const int64_t g = rp.offset + s;
                    const int64_t o4[4] = {
                        (i + 1 < (uint32_t)rp.n0) ? (int64_t)n12 : -(int64_t)(rp.n0 - 1) * n12,
                        (i > 0) ? -(int64_t)n12 : (int64_t)(rp.n0 - 1) * n12,
                        (j + 1 < (uint32_t)rp.n1) ? rp.n2 : -(int64_t)(rp.n1 - 1) * rp.n2,
                        (j > 0) ? -(int64_t)rp.n2 : (int64_t)(rp.n1 - 1) * rp.n2};
                    const int64_t gkr = g + ((k + 2 < (uint32_t)rp.n2) ? 2 : 2 - (int64_t)rp.n2);
                    const int64_t gkl = g + ((k > 0) ? -1 : (int64_t)(rp.n2 - 1));
                    const float* base[4] = {phi, phi + N, pi, pi + N};  // phi hi, lo, pi hi, lo
                    float2 dsum[4], cen[4];
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        const float* b = base[f];
                        const float2 cc = __ldg(reinterpret_cast<const float2*>(b + g));
                        float2 nb[6];
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            nb[u] = __ldg(reinterpret_cast<const float2*>(b + g + o4[u]));
                        const float kr = __ldg(b + gkr), kl = __ldg(b + gkl);  // k+1, k-1
                        // the order of stencil_sums_k: i and j terms, then the k pair
                        float2 acc;
                        if ((f & 1) == 0) {  // hi: sum (hi_n - hi_c)
                            acc = v_add(v_sub(nb[0], cc), v_sub(nb[1], cc));
                            acc = v_add(acc, v_sub(nb[2], cc));
                            acc = v_add(acc, v_sub(nb[3], cc));
                            const float2 kk = make_float2(
                                __fadd_rn(__fsub_rn(cc.y, cc.x), __fsub_rn(kl, cc.x)),
                                __fadd_rn(__fsub_rn(kr, cc.y), __fsub_rn(cc.x, cc.y)));
                            acc = v_add(acc, kk);
                        } else {             // lo: fma(-6, lo_c, sum lo_n)
                            acc = v_add(v_add(v_add(nb[0], nb[1]), nb[2]), nb[3]);
                            const float2 kk = make_float2(__fadd_rn(cc.y, kl), __fadd_rn(kr, cc.x));
                            acc = v_fma(vs<float2>(-6.0f), cc, v_add(acc, kk));
                        }
                        dsum[f] = acc;
                        cen[f] = cc;
                    }
                    F32CIn<float2> x;
                    x.dh_phi = dsum[0];
                    x.dl_phi = dsum[1];
                    x.dh_pi = dsum[2];
                    x.dl_pi = dsum[3];
                    x.phh = cen[0];
                    x.phl = cen[1];
                    x.pih = cen[2];
                    x.pil = cen[3];
                    float2 a, b, cc, d;
                    update_f32c<float2, false>(p, kc, nullptr, x, site_kick_f32c2(p, kc, (uint64_t)s), a, b,
                                        cc, d);
                    *reinterpret_cast<float2*>(po + g) = a;
                    *reinterpret_cast<float2*>(po + N + g) = b;
                    *reinterpret_cast<float2*>(vo + g) = cc;
                    *reinterpret_cast<float2*>(vo + N + g) = d;
                }
                continue;
            }
        }
        for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
            const uint32_t s = (uint32_t)(ch.begin + t);
            const uint32_t q = fdiv(s, rp.m2);
            const uint32_t k = s - q * (uint32_t)rp.n2;
            const uint32_t i = fdiv(q, rp.m1);
            const uint32_t j = q - i * (uint32_t)rp.n1;
            const int64_t o_ip = (i + 1 < (uint32_t)rp.n0) ? (int64_t)n12 : -(int64_t)(rp.n0 - 1) * n12;
            const int64_t o_im = (i > 0) ? -(int64_t)n12 : (int64_t)(rp.n0 - 1) * n12;
            const int64_t o_jp = (j + 1 < (uint32_t)rp.n1) ? rp.n2 : -(int64_t)(rp.n1 - 1) * rp.n2;
            const int64_t o_jm = (j > 0) ? -(int64_t)rp.n2 : (int64_t)(rp.n1 - 1) * rp.n2;
            const int64_t o_kp = (k + 1 < (uint32_t)rp.n2) ? 1 : -(int64_t)(rp.n2 - 1);
            const int64_t o_km = (k > 0) ? -1 : (int64_t)(rp.n2 - 1);
            const int64_t g = rp.offset + s;
            const int64_t idx[7] = {g, g + o_ip, g + o_im, g + o_jp, g + o_jm, g + o_kp, g + o_km};
            if constexpr (S == TIPT_F64) {
                const double* phi = static_cast<const double*>(e.phi);
                const double* pi = static_cast<const double*>(e.pi);
                double ph[7], pv[7];
#pragma unroll
                for (int u = 0; u < 7; ++u) {
                    ph[u] = __ldg(phi + idx[u]);
                    pv[u] = __ldg(pi + idx[u]);
                }
                double a, b;
                update_f64<false>(p, nullptr, ph, pv, site_noise<double>(p, (uint64_t)s), a, b);
                static_cast<double*>(e.phi_out)[g] = a;
                static_cast<double*>(e.pi_out)[g] = b;
            } else {
                const float* phi = static_cast<const float*>(e.phi);
                const float* pi = static_cast<const float*>(e.pi);
                const int64_t N = e.n_total;
                float hh[7], hl[7], vh[7], vl[7];
#pragma unroll
                for (int u = 0; u < 7; ++u) {
                    hh[u] = __ldg(phi + idx[u]);
                    hl[u] = __ldg(phi + N + idx[u]);
                    vh[u] = __ldg(pi + idx[u]);
                    vl[u] = __ldg(pi + N + idx[u]);
                }
                F32CIn<float> x;
                stencil_sums_k(hh, hl, x.dh_phi, x.dl_phi);
                stencil_sums_k(vh, vl, x.dh_pi, x.dl_pi);
                x.phh = hh[0];
                x.phl = hl[0];
                x.pih = vh[0];
                x.pil = vl[0];
                float a, b, cc, d;
                update_f32c<float, false>(p, kc, nullptr, x, site_kick_f32c(p, kc, (uint64_t)s), a, b,
                                   cc, d);
                float* po = static_cast<float*>(e.phi_out);
                float* vo = static_cast<float*>(e.pi_out);
                po[g] = a;
                po[N + g] = b;
                vo[g] = cc;
                vo[N + g] = d;
            }
        }
    }
}

// One block per replica: fraction of sites with phi > thr in a fixed order.
template <int S>
__global__ void __launch_bounds__(256) ensemble_observe_kernel(
    const void* phi, int64_t n_total, const tipt_replica* reps, int32_t* active,
    int32_t* n_active, double thr, double stop_frac, double retire_frac, uint64_t step0,
    const unsigned long long* ctr, long long offset, int64_t* first_step, double* frac_out) {
    __shared__ double s_part[256];
    const uint64_t step = step0 + (ctr ? *ctr + (unsigned long long)offset : 0ull);
    const int r = blockIdx.x;
    const tipt_replica rp = reps[r];
    const int64_t n = (int64_t)rp.n0 * rp.n1 * rp.n2;
    double cnt = 0.0;
    for (int64_t s = threadIdx.x; s < n; s += blockDim.x) {
        const int64_t g = rp.offset + s;
        double v;
        if constexpr (S == TIPT_F64) v = static_cast<const double*>(phi)[g];
        else {
            const float* f = static_cast<const float*>(phi);
            v = (double)f[g] + (double)f[n_total + g];
        }
        cnt += v > thr ? 1.0 : 0.0;
    }
    s_part[threadIdx.x] = cnt;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s_part[threadIdx.x] += s_part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double frac = s_part[0] / (double)n;
        frac_out[r] = frac;
        if (active[r]) {
            if (frac > stop_frac && first_step[r] < 0) first_step[r] = (int64_t)step;
            if (frac > retire_frac) {
                active[r] = 0;
                atomicSub(n_active, 1);
            }
        }
    }
}

}  // namespace tipt

using namespace tipt;

extern "C" int tipt_ensemble_step(int storage, const void* phi, const void* pi, void* phi_out,
                                  void* pi_out, int64_t n_total, const tipt_replica* replicas,
                                  const tipt_chunk* chunks, int32_t n_chunks,
                                  const int32_t* active, const tipt_step_params* sp,
                                  const uint64_t* counter, int64_t offset, void* stream) {
    int rc;
    if (storage != TIPT_F64 && storage != TIPT_F32C)
        return fail(TIPT_ERR_STORAGE, "the ensemble takes F64 or F32C storage");
    if ((rc = check_state_sites(storage, phi, pi, phi_out, pi_out, n_total))) return rc;
    if (!replicas || !chunks || !active || !sp) return fail(TIPT_ERR_ARG, "NULL argument");
    if (n_chunks < 0) return fail(TIPT_ERR_ARG, "n_chunks < 0");
    if (n_chunks == 0) return TIPT_OK;
    EnsParams e;
    e.phi = phi;
    e.pi = pi;
    e.phi_out = phi_out;
    e.pi_out = pi_out;
    e.n_total = n_total;
    e.reps = replicas;
    e.chunks = chunks;
    e.n_chunks = n_chunks;
    e.active = active;
    e.h1 = 0.5 * sp->dt;
    e.h2 = sp->dt;
    e.inv_dx2 = 1.0 / (sp->dx * sp->dx);
    e.eta = sp->eta_eff;
    e.inv_mu2 = 1.0 / (sp->mu * sp->mu);
    e.inv_a2 = sp->inv_a2;
    e.step = sp->noise_step;
    e.ctr = reinterpret_cast<const unsigned long long*>(counter);
    e.offset = offset;
    int grid = num_sms() * 8;
    if (grid > n_chunks) grid = n_chunks;
    cudaStream_t st = (cudaStream_t)stream;
    if (storage == TIPT_F64) ensemble_stage_kernel<TIPT_F64><<<grid, 256, 0, st>>>(e);
    else ensemble_stage_kernel<TIPT_F32C><<<grid, 256, 0, st>>>(e);
    cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? TIPT_OK : fail_cuda(err, "ensemble_stage launch");
}

extern "C" int tipt_ensemble_observe(int storage, const void* phi, int64_t n_total,
                                     const tipt_replica* replicas, int32_t n_replicas,
                                     int32_t* active, int32_t* n_active, double thr,
                                     double stop_frac, double retire_frac, uint64_t step,
                                     const uint64_t* counter,
                                     int64_t offset, int64_t* first_step, double* frac_out,
                                     void* stream) {
    if (storage != TIPT_F64 && storage != TIPT_F32C)
        return fail(TIPT_ERR_STORAGE, "the ensemble takes F64 or F32C storage");
    if (!phi || !replicas || !active || !n_active || !first_step || !frac_out)
        return fail(TIPT_ERR_ARG, "NULL argument");
    if (!(retire_frac >= stop_frac))
        return fail(TIPT_ERR_ARG, "retire_frac must be >= stop_frac");
    if (n_replicas <= 0) return TIPT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (storage == TIPT_F64)
        ensemble_observe_kernel<TIPT_F64><<<n_replicas, 256, 0, st>>>(
            phi, n_total, replicas, active, n_active, thr, stop_frac, retire_frac, step,
            reinterpret_cast<const unsigned long long*>(counter), offset, first_step, frac_out);
    else
        ensemble_observe_kernel<TIPT_F32C><<<n_replicas, 256, 0, st>>>(
            phi, n_total, replicas, active, n_active, thr, stop_frac, retire_frac, step,
            reinterpret_cast<const unsigned long long*>(counter), offset, first_step, frac_out);
    cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? TIPT_OK : fail_cuda(err, "ensemble_observe launch");
}

// The replicas of one 3-D shape class in compensated FP32 on the marching stage
// (shared-memory tiles, TMA/bulk-copy ring): bitwise the same step as
// tipt_ensemble_step for those replicas.
extern "C" int tipt_ensemble_step_march(const void* phi, const void* pi, void* phi_out,
                                        void* pi_out, int64_t n_total,
                                        const tipt_replica* replicas, const int32_t* rids,
                                        int32_t n_rids, const int32_t* n_rids_dev, int32_t n0,
                                        int32_t n1, int32_t n2, const int32_t* active,
                                        const tipt_step_params* sp, const uint64_t* counter,
                                        int64_t offset, void* stream) {
    int rc;
    if ((rc = check_state_sites(TIPT_F32C, phi, pi, phi_out, pi_out, n_total))) return rc;
    if (!replicas || !rids || !active || !sp) return fail(TIPT_ERR_ARG, "NULL argument");
    if (n_rids < 0) return fail(TIPT_ERR_ARG, "n_rids < 0");
    if (n_rids == 0) return TIPT_OK;
    if (!ensemble_march_supported(n0, n1, n2))
        return fail(TIPT_ERR_UNSUPPORTED, "replica shape %d x %d x %d has no marching tiles", n0,
                    n1, n2);
    const uintptr_t a = reinterpret_cast<uintptr_t>(phi) | reinterpret_cast<uintptr_t>(pi) |
                        reinterpret_cast<uintptr_t>(phi_out) | reinterpret_cast<uintptr_t>(pi_out);
    if (a % 16 || (n_total * 4) % 16) return fail(TIPT_ERR_ALIGN, "packed buffers must be 16-byte aligned");
    RealStageParams p;
    memset(&p, 0, sizeof(p));
    p.phi = phi;
    p.pi = pi;
    p.phi_out = phi_out;
    p.pi_out = pi_out;
    p.n0 = n0;
    p.n1 = n1;
    p.n2 = n2;
    p.h1 = 0.5 * sp->dt;
    p.h2 = sp->dt;
    p.inv_dx2 = 1.0 / (sp->dx * sp->dx);
    p.eta = sp->eta_eff;
    p.inv_mu2 = 1.0 / (sp->mu * sp->mu);
    p.inv_a2 = sp->inv_a2;
    p.nfac = 1.0;
    p.step = sp->noise_step;
    return launch_ensemble_march(p, replicas, rids, n_rids, n_rids_dev, active, n_total,
                                 reinterpret_cast<const unsigned long long*>(counter),
                                 (long long)offset, (cudaStream_t)stream);
}

// 1 when replicas of shape n0 x n1 x n2 (n2 contiguous) can step on the marching
// stage (tipt_ensemble_step_march), 0 otherwise.
extern "C" int tipt_ensemble_march_supported(int32_t n0, int32_t n1, int32_t n2) {
    return ensemble_march_supported(n0, n1, n2) ? 1 : 0;
}

// Ordered compaction of a class's replica ids: rids_out[0..*n_out) = the ids
// rids[q] (in order) whose active flag is set.  One block.
__global__ void __launch_bounds__(1024) ensemble_compact_kernel(const int32_t* rids, int32_t n,
                                                                 const int32_t* active,
                                                                 int32_t* rids_out,
                                                                 int32_t* n_out) {
    __shared__ int32_t s_warp[32];
    __shared__ int32_t s_base;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int b = 0; b < n; b += blockDim.x) {
        const int q = b + (int)threadIdx.x;
        const bool keep = q < n && active[rids[q]] != 0;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_warp[wid] = __popc(m);
        __syncthreads();
        int before = s_base;
        for (int w = 0; w < wid; ++w) before += s_warp[w];
        if (keep) rids_out[before + __popc(m & ((1u << lane) - 1u))] = rids[q];
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s_warp[w];
            s_base += tot;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *n_out = s_base;
}

// The active replicas of a class, compacted in order (for tipt_ensemble_step_march's
// device count): rids_out receives them, *n_out their number.
extern "C" int tipt_ensemble_compact(const int32_t* rids, int32_t n, const int32_t* active,
                                     int32_t* rids_out, int32_t* n_out, void* stream) {
    if (!rids || !active || !rids_out || !n_out) return fail(TIPT_ERR_ARG, "NULL argument");
    if (n < 0) return fail(TIPT_ERR_ARG, "n < 0");
    ensemble_compact_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(rids, n, active, rids_out,
                                                                  n_out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "ensemble_compact launch");
}
