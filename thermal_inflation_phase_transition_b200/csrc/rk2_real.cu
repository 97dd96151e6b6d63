// Real-field fused midpoint RK2 stage kernels.
//
//  * rk2_stage_generic: one site per thread (grid-stride), any lattice shape
//    and storage; loads the 7-point stencil of phi and pi straight from HBM
//    through L1.  Used for shapes the marching kernel does not cover.
//  * rk2_stage_march (rk2_march.cuh): the bandwidth kernel for n2 % 4 == 0.
#include "rk2_real.cuh"
#include "rk2_march.cuh"
#include "tipt_internal.h"

namespace tipt {

template <int S, bool TH, bool RG>
__global__ void __launch_bounds__(256) rk2_stage_generic(RealStageParams p_in) {
    RealStageParams p = p_in;
    resolve_schedule(p);
    if constexpr (RG) reset_next_range(p);
    RangeAcc racc;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using TT = typename std::conditional<S == TIPT_F32C, float, double>::type;
    TT* s_tab = reinterpret_cast<TT*>(smem_raw);
    if (p.table_in_smem) stage_table<TT>(p, s_tab);
    const F32CConst kc = f32c_const(p);

    const int64_t n12 = (int64_t)p.n1 * p.n2;
    const int64_t N = (int64_t)p.n0 * n12;
    const int64_t s_end = (int64_t)p.i_end * n12;
    for (int64_t s = (int64_t)p.i_begin * n12 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
         s < s_end; s += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(s % p.n2);
        const int64_t r = s / p.n2;
        const int j = (int)(r % p.n1);
        const int i = (int)(r / p.n1);
        const int64_t o_ip = (i + 1 < p.n0) ? n12 : -(int64_t)(p.n0 - 1) * n12;
        const int64_t o_im = (i > 0) ? -n12 : (int64_t)(p.n0 - 1) * n12;
        const int64_t o_jp = (j + 1 < p.n1) ? p.n2 : -(int64_t)(p.n1 - 1) * p.n2;
        const int64_t o_jm = (j > 0) ? -(int64_t)p.n2 : (int64_t)(p.n1 - 1) * p.n2;
        const int64_t o_kp = (k + 1 < p.n2) ? 1 : -(int64_t)(p.n2 - 1);
        const int64_t o_km = (k > 0) ? -1 : (int64_t)(p.n2 - 1);
        const int64_t idx[7] = {s, s + o_ip, s + o_im, s + o_jp, s + o_jm, s + o_kp, s + o_km};
        if constexpr (S == TIPT_F64) {
            const double* phi = static_cast<const double*>(p.phi);
            const double* pi = static_cast<const double*>(p.pi);
            double ph[7], pv[7];
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                ph[q] = __ldg(phi + idx[q]);
                pv[q] = __ldg(pi + idx[q]);
            }
            double a, b;
            update_f64<TH>(p, reinterpret_cast<const double*>(s_tab), ph, pv,
                       site_noise<double>(p, (uint64_t)(s + p.site_offset)), a, b);
            static_cast<double*>(p.phi_out)[s] = a;
            static_cast<double*>(p.pi_out)[s] = b;
            if constexpr (RG) racc.fold_d(a);
        } else if constexpr (S == TIPT_F32) {
            const float* phi = static_cast<const float*>(p.phi);
            const float* pi = static_cast<const float*>(p.pi);
            float ph[7], pv[7];
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                ph[q] = __ldg(phi + idx[q]);
                pv[q] = __ldg(pi + idx[q]);
            }
            float a, b;
            update_f32<TH>(p, reinterpret_cast<const double*>(s_tab), ph, pv,
                       site_noise<float>(p, (uint64_t)(s + p.site_offset)), a, b);
            static_cast<float*>(p.phi_out)[s] = a;
            static_cast<float*>(p.pi_out)[s] = b;
            if constexpr (RG) racc.fold(a);
        } else {
            // planar {hi, lo}: hi plane at [0, N), lo plane at [N, 2N)
            const float* phi = static_cast<const float*>(p.phi);
            const float* pi = static_cast<const float*>(p.pi);
            float hh[7], hl[7], vh[7], vl[7];
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                hh[q] = __ldg(phi + idx[q]);
                hl[q] = __ldg(phi + N + idx[q]);
                vh[q] = __ldg(pi + idx[q]);
                vl[q] = __ldg(pi + N + idx[q]);
            }
            F32CIn<float> x;
            stencil_sums_k(hh, hl, x.dh_phi, x.dl_phi);
            stencil_sums_k(vh, vl, x.dh_pi, x.dl_pi);
            x.phh = hh[0];
            x.phl = hl[0];
            x.pih = vh[0];
            x.pil = vl[0];
            float a, b, c, d;
            update_f32c<float, TH>(p, kc, reinterpret_cast<const float*>(s_tab), x,
                               site_kick_f32c(p, kc, (uint64_t)(s + p.site_offset)), a, b, c, d);
            float* po = static_cast<float*>(p.phi_out);
            float* vo = static_cast<float*>(p.pi_out);
            po[s] = a;
            po[N + s] = b;
            vo[s] = c;
            vo[N + s] = d;
            if constexpr (RG) racc.fold_ff(a, b);
        }
    }
    if constexpr (RG) racc.flush(p.range);
}

// Bytes of shared memory the V' row needs for storage S (0 if polynomial).
static int64_t table_smem_bytes(int S, const RealStageParams& p) {
    if (p.vkind == TIPT_VP_POLY || p.vkind == TIPT_VP_THERMAL) return 0;
    return (int64_t)p.npts * (S == TIPT_F32C ? 4 : 8);
}

static int g_num_sms = 0;
int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

template <int S>
static int launch_generic(RealStageParams p, int64_t smem, cudaStream_t st) {
    auto kern = p.vkind == TIPT_VP_THERMAL
                    ? (p.range ? rk2_stage_generic<S, true, true> : rk2_stage_generic<S, true, false>)
                    : (p.range ? rk2_stage_generic<S, false, true> : rk2_stage_generic<S, false, false>);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return fail_cuda(e, "rk2_stage_generic smem attribute");
    }
    const int64_t N = (int64_t)(p.i_end - p.i_begin) * p.n1 * p.n2;
    int64_t blocks = (N + 255) / 256;
    const int64_t cap = (int64_t)num_sms() * 8;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, 256, (size_t)smem, st>>>(p);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "rk2_stage_generic launch");
}

// Largest V' row staged in shared memory; longer 1-D tables are read from
// global memory (L1/L2 resident), longer 2-D tables are rejected.
constexpr int64_t kMaxTableSmem = 96 * 1024;

// Kernel choice: 0 automatic, 1 generic kernel only, 2 marching kernel only.
static int g_kernel_policy = 0;

int kernel_policy() { return g_kernel_policy; }

// A lattice whose contiguous extent is 1 (the reference's 2-D form nz = 1) is
// relabelled so the contiguous axis is the longest non-trivial one: (nx, ny, 1)
// -> (1, nx, ny) and (nx, 1, 1) -> (1, 1, nx).  Linear site indices, hence the
// noise keys, are unchanged; the neighbour set of every site is the same.
static void canonical_shape(RealStageParams& p) {
    if (p.n2 != 1) return;
    if (p.n1 > 1) {
        p.n2 = p.n1;
        p.n1 = p.n0;
        p.n0 = 1;
    } else {
        p.n2 = p.n0;
        p.n0 = 1;
    }
}

int launch_real_stage(int storage, RealStageParams p, cudaStream_t st) {
    if (p.i_end == 0) {
        canonical_shape(p);
        p.i_begin = 0;
        p.i_end = p.n0;
    }
    const int64_t tb = table_smem_bytes(storage, p);
    p.table_in_smem = (tb > 0 && tb <= kMaxTableSmem) ? 1 : 0;
    if (p.vkind == TIPT_VP_TABLE2D && !p.table_in_smem)
        return fail(TIPT_ERR_UNSUPPORTED, "2-D V' table row of %d points exceeds %lld bytes of "
                    "shared memory", p.npts, (long long)kMaxTableSmem);
    const int64_t smem = p.table_in_smem ? tb : 0;
    set_f32c_pairs(p);
    const bool march = g_kernel_policy != 1 && march_supported(storage, p);
    if (g_kernel_policy == 2 && !march)
        return fail(TIPT_ERR_UNSUPPORTED, "marching kernel does not cover this shape/storage");
    if (march) return launch_march(storage, p, smem, st);
    switch (storage) {
        case TIPT_F64: return launch_generic<TIPT_F64>(p, smem, st);
        case TIPT_F32: return launch_generic<TIPT_F32>(p, smem, st);
        case TIPT_F32C: return launch_generic<TIPT_F32C>(p, smem, st);
    }
    return fail(TIPT_ERR_STORAGE, "unknown storage %d", storage);
}

}  // namespace tipt

// Selects the real-field stage kernel: 0 automatic (the marching kernel where it
// applies), 1 the generic kernel, 2 the marching kernel or an error.  Results are
// bitwise identical between the two kernels; this exists for tests and tuning.
extern "C" int tipt_set_kernel_policy(int policy) {
    if (policy < 0 || policy > 2) return tipt::fail(TIPT_ERR_ARG, "policy must be 0, 1 or 2");
    tipt::g_kernel_policy = policy;
    return TIPT_OK;
}
