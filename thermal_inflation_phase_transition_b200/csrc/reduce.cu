// Observable reductions: compute_energy_densities (R:2270-2319) plus <phi>,
// <phi^2>, <pi^2>, the converted fraction, min/max and the non-finite count
// of the host NaN guard (R:3882-3944).
//
// Two launches, both deterministic: (1) a fixed number of blocks G (a
// function of the lattice size only) each reduce a contiguous range of
// sites with warp shuffles into FP64 partials in the caller's workspace;
// (2) one block folds the G partials in a fixed order.  The result does not
// depend on the GPU or on timing.
#include "tipt_device.cuh"
#include "tipt_internal.h"

namespace tipt {

constexpr int kObs = 10;          // outputs
constexpr int kRedThreads = 256;
constexpr int kMaxRedBlocks = 1184;

// Accumulators: grad = sum of squared forward differences (the constants 0.5
// inv_a2 inv_dx2 are applied once at the end), sq = sum of pi^2 (E_kin = sq / 2,
// bitwise the sum of pi^2 / 2: halving commutes with FP64 rounding).
struct ObsAcc {
    double grad, pot, s1, s2, sq, above, nonfinite, mn, mx;
};

__device__ __forceinline__ void acc_init(ObsAcc& a) {
    a.grad = a.pot = a.s1 = a.s2 = a.sq = a.above = a.nonfinite = 0.0;
    a.mn = INFINITY;
    a.mx = -INFINITY;
}

__device__ __forceinline__ void acc_merge(ObsAcc& a, const ObsAcc& b) {
    a.grad += b.grad;
    a.pot += b.pot;
    a.s1 += b.s1;
    a.s2 += b.s2;
    a.sq += b.sq;
    a.above += b.above;
    a.nonfinite += b.nonfinite;
    a.mn = fmin(a.mn, b.mn);
    a.mx = fmax(a.mx, b.mx);
}

__device__ __forceinline__ ObsAcc acc_shfl_down(const ObsAcc& a, int off) {
    ObsAcc b;
    b.grad = __shfl_down_sync(0xffffffffu, a.grad, off);
    b.pot = __shfl_down_sync(0xffffffffu, a.pot, off);
    b.s1 = __shfl_down_sync(0xffffffffu, a.s1, off);
    b.s2 = __shfl_down_sync(0xffffffffu, a.s2, off);
    b.sq = __shfl_down_sync(0xffffffffu, a.sq, off);
    b.above = __shfl_down_sync(0xffffffffu, a.above, off);
    b.nonfinite = __shfl_down_sync(0xffffffffu, a.nonfinite, off);
    b.mn = __shfl_down_sync(0xffffffffu, a.mn, off);
    b.mx = __shfl_down_sync(0xffffffffu, a.mx, off);
    return b;
}

// Block-wide fixed-order reduction; result valid in thread 0.
__device__ __forceinline__ ObsAcc block_reduce(ObsAcc a) {
    __shared__ ObsAcc s_w[kRedThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc_merge(a, acc_shfl_down(a, off));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) s_w[w] = a;
    __syncthreads();
    if (w == 0) {
        if (l < kRedThreads / 32) a = s_w[l];
        else acc_init(a);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc_merge(a, acc_shfl_down(a, off));
    }
    return a;
}

// Site value in FP64; F32C is planar (hi plane, then lo plane N sites later).
template <int S>
__device__ __forceinline__ double load_val(const void* p, int64_t s, int64_t N) {
    if constexpr (S == TIPT_F64) return __ldg(static_cast<const double*>(p) + s);
    else if constexpr (S == TIPT_F32) return (double)__ldg(static_cast<const float*>(p) + s);
    else {
        const float* f = static_cast<const float*>(p);
        return (double)__ldg(f + s) + (double)__ldg(f + N + s);
    }
}

struct ObsParams {
    const void* phi;
    const void* pi;
    int n0, n1, n2;
    int i_begin, i_end;  // planes reduced (the i+1 neighbour of the last may lie outside)
    double inv_dx2, inv_a2, lam, m2, inv_mu2, thr;
    double* partials;  // [G][kObs]
    double* out;       // [kObs]
};

// Sites are walked row by row (a row = the n2 sites of fixed (i, j)): warp w
// of block b takes rows w + 8 b, w + 8 b + 8 G, ... and its lanes stride along
// the row, so loads are coalesced and the only divisions are one 32-bit
// division per row.  The assignment depends on the lattice shape alone.
template <int S>
__device__ __forceinline__ void obs_site(const ObsParams& p, ObsAcc& a, int64_t s, int64_t ox,
                                         int64_t oy, int64_t oz, int64_t N) {
    const double ph = load_val<S>(p.phi, s, N);
    const double pv = p.pi ? load_val<S>(p.pi, s, N) : 0.0;
    // forward differences, R:2303-2308
    const double fx = load_val<S>(p.phi, s + ox, N) - ph;
    const double fy = load_val<S>(p.phi, s + oy, N) - ph;
    const double fz = load_val<S>(p.phi, s + oz, N) - ph;
    a.grad += fx * fx + fy * fy + fz * fz;
    const double ph2 = ph * ph;
    a.pot += (0.25 * p.lam * ph2 * ph2 - 0.5 * p.m2 * ph2) * p.inv_mu2;
    a.s1 += ph;
    a.s2 += ph2;
    a.sq += pv * pv;
    a.above += ph > p.thr ? 1.0 : 0.0;
    a.nonfinite += (isfinite(ph) && isfinite(pv)) ? 0.0 : 1.0;
    a.mn = fmin(a.mn, ph);
    a.mx = fmax(a.mx, ph);
}

template <int S>
__global__ void __launch_bounds__(kRedThreads) obs_partial_kernel(ObsParams p) {
    const int64_t n12 = (int64_t)p.n1 * p.n2;
    const int64_t N = (int64_t)p.n0 * n12;
    const int64_t rows = (int64_t)p.i_end * p.n1;
    const int lane = threadIdx.x & 31;
    const int wpb = kRedThreads / 32;
    ObsAcc a;
    acc_init(a);
    for (int64_t row = (int64_t)p.i_begin * p.n1 + (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5);
         row < rows; row += (int64_t)gridDim.x * wpb) {
        const int64_t i = row / p.n1;
        const int64_t j = row - i * p.n1;
        const int64_t ox = (i + 1 < p.n0) ? n12 : -(int64_t)(p.n0 - 1) * n12;
        const int64_t oy = (j + 1 < p.n1) ? (int64_t)p.n2 : -(int64_t)(p.n1 - 1) * p.n2;
        const int64_t base = row * p.n2;
        int k = lane;
        // two sites per lane per pass keep more loads in flight
        for (; k + 32 < p.n2; k += 64) {
            obs_site<S>(p, a, base + k, ox, oy, 1, N);
            obs_site<S>(p, a, base + k + 32, ox, oy, (k + 33 < p.n2) ? 1 : -(int64_t)(p.n2 - 1), N);
        }
        if (k < p.n2) obs_site<S>(p, a, base + k, ox, oy, (k + 1 < p.n2) ? 1 : -(int64_t)(p.n2 - 1), N);
    }
    a = block_reduce(a);
    if (threadIdx.x == 0) {
        double* o = p.partials + (int64_t)blockIdx.x * kObs;
        o[0] = 0.0;  // slot kept so the workspace layout stays [G][kObs]
        o[1] = a.grad;
        o[2] = a.pot;
        o[3] = a.s1;
        o[4] = a.s2;
        o[5] = a.sq;
        o[6] = a.above;
        o[7] = a.mn;
        o[8] = a.mx;
        o[9] = a.nonfinite;
    }
}

// Marching form for n2 % 4 == 0 (the bandwidth path).  A thread owns four
// consecutive sites (j, k0..k0+3) of a row and walks a chunk of kObsPlanes
// planes along i: plane i+1 is its i-neighbour and next centre, so every value
// is read from memory once (the j+1 row and the k0+4 site come from the
// neighbouring threads' reads through L1).  Block (x, y) reduces the 256
// threads of column group x over plane chunk y; the partition depends on the
// shape only.
constexpr int kObsPlanes = 64;

// Four consecutive sites as FP64 (F64 and F32 storages; compensated FP32 has
// its own kernel below).
template <int S>
__device__ __forceinline__ void load4(const void* f, int64_t s, double v[4]) {
    if constexpr (S == TIPT_F64) {
        const double2* q = reinterpret_cast<const double2*>(static_cast<const double*>(f) + s);
        const double2 a = __ldg(q), b = __ldg(q + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else {
        static_assert(S == TIPT_F32, "F64 or F32 storage");
        const float4 a = __ldg(reinterpret_cast<const float4*>(static_cast<const float*>(f) + s));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
}

template <int S>
__global__ void __launch_bounds__(kRedThreads) obs_march_kernel(ObsParams p) {
    const int n0 = p.n0, n1 = p.n1, n2 = p.n2;
    const int64_t n12 = (int64_t)n1 * n2;
    const int64_t N = (int64_t)n0 * n12;
    const int tpr = n2 >> 2;
    const int64_t cols = (int64_t)n1 * tpr;
    const int64_t col = (int64_t)blockIdx.x * kRedThreads + threadIdx.x;
    ObsAcc a;
    acc_init(a);
    if (col < cols) {
        const int j = (int)(col / tpr);
        const int k0 = 4 * (int)(col - (int64_t)j * tpr);
        const int64_t rj = (int64_t)j * n2 + k0;                          // in-plane offset
        const int64_t rjp = (int64_t)(j + 1 < n1 ? j + 1 : 0) * n2 + k0;  // row j+1
        const int64_t rkp = (int64_t)j * n2 + (k0 + 4 < n2 ? k0 + 4 : 0); // site k0+4
        const int i0 = p.i_begin + blockIdx.y * kObsPlanes;
        const int ni = min(kObsPlanes, p.i_end - i0);
        double ph[4], pn[4], pv[4], jp[4], kp;
        load4<S>(p.phi, (int64_t)i0 * n12 + rj, ph);
        for (int q = 0; q < ni; ++q) {
            const int i = i0 + q;
            const int64_t pc = (int64_t)i * n12;
            const int64_t pnx = (int64_t)(i + 1 < n0 ? i + 1 : 0) * n12;
            load4<S>(p.phi, pnx + rj, pn);
            load4<S>(p.phi, pc + rjp, jp);
            if (p.pi) load4<S>(p.pi, pc + rj, pv);
            else pv[0] = pv[1] = pv[2] = pv[3] = 0.0;
            kp = load_val<S>(p.phi, pc + rkp, N);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const double c = ph[u];
                // forward differences, R:2303-2308
                const double fx = pn[u] - c;
                const double fy = jp[u] - c;
                const double fz = (u < 3 ? ph[u + 1] : kp) - c;
                a.grad += fx * fx + fy * fy + fz * fz;
                const double c2 = c * c;
                a.pot += (0.25 * p.lam * c2 * c2 - 0.5 * p.m2 * c2) * p.inv_mu2;
                a.s1 += c;
                a.s2 += c2;
                a.sq += pv[u] * pv[u];
                a.above += c > p.thr ? 1.0 : 0.0;
                a.nonfinite += (isfinite(c) && isfinite(pv[u])) ? 0.0 : 1.0;
                a.mn = fmin(a.mn, c);
                a.mx = fmax(a.mx, c);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) ph[u] = pn[u];
        }
    }
    a = block_reduce(a);
    if (threadIdx.x == 0) {
        double* o = p.partials + ((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * kObs;
        o[0] = 0.0;
        o[1] = a.grad;
        o[2] = a.pot;
        o[3] = a.s1;
        o[4] = a.s2;
        o[5] = a.sq;
        o[6] = a.above;
        o[7] = a.mn;
        o[8] = a.mx;
        o[9] = a.nonfinite;
    }
}

// Compensated-FP32 form of the marching reduction: the per-site terms in FP32
// -- a value as hi + lo, a neighbour difference as (hi_n - hi_c) + (lo_n - lo_c)
// (the hi difference is exact for close neighbours) -- summed over the
// thread's four sites in FP32 and added to the FP64 accumulators once per
// plane (a term's relative error is about 6e-8; min and max are FP32 values of
// hi + lo).  The threshold test compares the pair with the threshold split
// into hi + lo, so it is exact.
__global__ void __launch_bounds__(kRedThreads) obs_march_f32c_kernel(ObsParams p) {
    const int n0 = p.n0, n1 = p.n1, n2 = p.n2;
    const int64_t n12 = (int64_t)n1 * n2;
    const int64_t N = (int64_t)n0 * n12;
    const int tpr = n2 >> 2;
    const int64_t cols = (int64_t)n1 * tpr;
    const int64_t col = (int64_t)blockIdx.x * kRedThreads + threadIdx.x;
    ObsAcc a;
    acc_init(a);
    if (col < cols) {
        const float* phi = static_cast<const float*>(p.phi);
        const float* pi = static_cast<const float*>(p.pi);
        const int j = (int)(col / tpr);
        const int k0 = 4 * (int)(col - (int64_t)j * tpr);
        const int64_t rj = (int64_t)j * n2 + k0;
        const int64_t rjp = (int64_t)(j + 1 < n1 ? j + 1 : 0) * n2 + k0;
        const int64_t rkp = (int64_t)j * n2 + (k0 + 4 < n2 ? k0 + 4 : 0);
        const int i0 = p.i_begin + blockIdx.y * kObsPlanes;
        const int ni = min(kObsPlanes, p.i_end - i0);
        const float qa = (float)(0.25 * p.lam), qb = (float)(-0.5 * p.m2);
        const float th = (float)p.thr, tl = (float)(p.thr - (double)th);
        auto ld4 = [&](const float* f, int64_t o, float v[4]) {
            const float4 x = __ldg(reinterpret_cast<const float4*>(f + o));
            v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
        };
        float ch[4], cl[4];
        ld4(phi, (int64_t)i0 * n12 + rj, ch);
        ld4(phi, N + (int64_t)i0 * n12 + rj, cl);
        for (int q = 0; q < ni; ++q) {
            const int i = i0 + q;
            const int64_t pc = (int64_t)i * n12;
            const int64_t pnx = (int64_t)(i + 1 < n0 ? i + 1 : 0) * n12;
            float nh[4], nl[4], jh[4], jl[4], vh[4] = {0, 0, 0, 0}, vl[4] = {0, 0, 0, 0};
            ld4(phi, pnx + rj, nh);
            ld4(phi, N + pnx + rj, nl);
            ld4(phi, pc + rjp, jh);
            ld4(phi, N + pc + rjp, jl);
            if (pi) {
                ld4(pi, pc + rj, vh);
                ld4(pi, N + pc + rj, vl);
            }
            const float kh = __ldg(phi + pc + rkp), kl = __ldg(phi + N + pc + rkp);
            float gs = 0.0f, ps = 0.0f, s1 = 0.0f, s2 = 0.0f, sq = 0.0f;
            float mn = INFINITY, mx = -INFINITY;
            int above = 0, bad = 0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float c = __fadd_rn(ch[u], cl[u]);
                // forward differences, R:2303-2308
                const float fx = __fadd_rn(__fsub_rn(nh[u], ch[u]), __fsub_rn(nl[u], cl[u]));
                const float fy = __fadd_rn(__fsub_rn(jh[u], ch[u]), __fsub_rn(jl[u], cl[u]));
                const float fz = __fadd_rn(__fsub_rn(u < 3 ? ch[u + 1] : kh, ch[u]),
                                           __fsub_rn(u < 3 ? cl[u + 1] : kl, cl[u]));
                gs = __fmaf_rn(fx, fx, __fmaf_rn(fy, fy, __fmaf_rn(fz, fz, gs)));
                const float c2 = __fmul_rn(c, c);
                ps = __fmaf_rn(__fmaf_rn(qa, c2, qb), c2, ps);
                s1 = __fadd_rn(s1, c);
                s2 = __fadd_rn(s2, c2);
                const float v = __fadd_rn(vh[u], vl[u]);
                sq = __fmaf_rn(v, v, sq);
                above += (ch[u] > th || (ch[u] == th && cl[u] > tl)) ? 1 : 0;
                bad += (isfinite(c) && isfinite(v)) ? 0 : 1;
                mn = fminf(mn, c);
                mx = fmaxf(mx, c);
            }
            a.grad += (double)gs;
            a.pot += (double)ps * p.inv_mu2;
            a.s1 += (double)s1;
            a.s2 += (double)s2;
            a.sq += (double)sq;
            a.above += (double)above;
            a.nonfinite += (double)bad;
            a.mn = fmin(a.mn, (double)mn);
            a.mx = fmax(a.mx, (double)mx);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                ch[u] = nh[u];
                cl[u] = nl[u];
            }
        }
    }
    a = block_reduce(a);
    if (threadIdx.x == 0) {
        double* o = p.partials + ((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * kObs;
        o[0] = 0.0;
        o[1] = a.grad;
        o[2] = a.pot;
        o[3] = a.s1;
        o[4] = a.s2;
        o[5] = a.sq;
        o[6] = a.above;
        o[7] = a.mn;
        o[8] = a.mx;
        o[9] = a.nonfinite;
    }
}

__global__ void __launch_bounds__(kRedThreads) obs_final_kernel(ObsParams p, int G, double inv_n) {
    ObsAcc a;
    acc_init(a);
    // fixed assignment: thread t folds partials t, t+256, ... in order
    for (int b = threadIdx.x; b < G; b += blockDim.x) {
        const double* o = p.partials + (int64_t)b * kObs;
        ObsAcc c;
        c.grad = o[1];
        c.pot = o[2];
        c.s1 = o[3];
        c.s2 = o[4];
        c.sq = o[5];
        c.above = o[6];
        c.mn = o[7];
        c.mx = o[8];
        c.nonfinite = o[9];
        acc_merge(a, c);
    }
    a = block_reduce(a);
    if (threadIdx.x == 0) {
        p.out[0] = 0.5 * a.sq * inv_n;
        p.out[1] = 0.5 * p.inv_a2 * p.inv_dx2 * a.grad * inv_n;
        p.out[2] = a.pot * inv_n;
        p.out[3] = a.s1 * inv_n;
        p.out[4] = a.s2 * inv_n;
        p.out[5] = a.sq * inv_n;
        p.out[6] = a.above * inv_n;
        p.out[7] = a.mn;
        p.out[8] = a.mx;
        p.out[9] = a.nonfinite;
    }
}

// Rows / 8 warps per block, at most kMaxRedBlocks (8 x 148): a function of the shape only.
int obs_blocks(int64_t rows) {
    int64_t g = (rows + 7) / 8;
    if (g > kMaxRedBlocks) g = kMaxRedBlocks;
    if (g < 1) g = 1;
    return (int)g;
}

// Grid of the marching form over n0 planes: (row groups of 256 four-site
// columns, plane chunks).
static bool obs_march_grid(int n0, int n1, int n2, dim3& grid) {
    if (n2 % 4 != 0 || n2 < 8) return false;
    const int64_t cols = (int64_t)n1 * (n2 / 4);
    const int64_t gx = (cols + kRedThreads - 1) / kRedThreads;
    const int64_t gy = (n0 + kObsPlanes - 1) / kObsPlanes;
    if (gx > 0x7fffffff || gy > 65535) return false;
    grid = dim3((unsigned)gx, (unsigned)gy, 1);
    return true;
}

int64_t obs_workspace_bytes(int n0, int n1, int n2) {
    int64_t g = obs_blocks((int64_t)n0 * n1);
    dim3 grid;
    if (obs_march_grid(n0, n1, n2, grid) && (int64_t)grid.x * grid.y > g)
        g = (int64_t)grid.x * grid.y;
    return g * kObs * 8;
}

// Reduces planes [i_begin, i_end) of an n0-plane array; means are taken over
// n_sites (the whole lattice, also when the array is one slab of it).
int launch_observables(int storage, const void* phi, const void* pi, int n0, int n1, int n2,
                       int i_begin, int i_end, double n_sites, double dx, double inv_a2,
                       double lam, double mphi, double mu, double thr, double* out,
                       double* partials, cudaStream_t st) {
    ObsParams p;
    p.phi = phi;
    p.pi = pi;
    p.n0 = n0;
    p.n1 = n1;
    p.n2 = n2;
    p.i_begin = i_begin;
    p.i_end = i_end;
    p.inv_dx2 = 1.0 / (dx * dx);
    p.inv_a2 = inv_a2;
    p.lam = lam;
    p.m2 = mphi * mphi;
    p.inv_mu2 = 1.0 / (mu * mu);
    p.thr = thr;
    p.partials = partials;
    p.out = out;
    const int planes = i_end - i_begin;
    int G = obs_blocks((int64_t)planes * n1);
    dim3 grid;
    const bool march = (reinterpret_cast<uintptr_t>(phi) | reinterpret_cast<uintptr_t>(pi)) % 16 == 0 &&
                       obs_march_grid(planes, n1, n2, grid);
    if (march) {
        G = (int)(grid.x * grid.y);
        switch (storage) {
            case TIPT_F64: obs_march_kernel<TIPT_F64><<<grid, kRedThreads, 0, st>>>(p); break;
            case TIPT_F32: obs_march_kernel<TIPT_F32><<<grid, kRedThreads, 0, st>>>(p); break;
            default: obs_march_f32c_kernel<<<grid, kRedThreads, 0, st>>>(p); break;
        }
    } else {
        switch (storage) {
            case TIPT_F64: obs_partial_kernel<TIPT_F64><<<G, kRedThreads, 0, st>>>(p); break;
            case TIPT_F32: obs_partial_kernel<TIPT_F32><<<G, kRedThreads, 0, st>>>(p); break;
            default: obs_partial_kernel<TIPT_F32C><<<G, kRedThreads, 0, st>>>(p); break;
        }
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "observables partial launch");
    obs_final_kernel<<<1, kRedThreads, 0, st>>>(p, G, 1.0 / n_sites);
    e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "observables final launch");
}

}  // namespace tipt

using namespace tipt;

extern "C" int64_t tipt_observables_workspace_size(int64_t nx, int64_t ny, int64_t nz) {
    if (nx < 1 || ny < 1 || nz < 1) return 0;
    // (nx, ny, 1) is walked as (1, nx, ny)
    if (nz == 1) return obs_workspace_bytes(1, (int)nx, (int)ny);
    return obs_workspace_bytes((int)nx, (int)ny, (int)nz);
}

extern "C" int tipt_observables(int storage, const void* phi, const void* pi, int64_t nx,
                                int64_t ny, int64_t nz, double dx, double inv_a2, double lam,
                                double mphi, double mu, double thr, double* out,
                                void* workspace, int64_t workspace_bytes, void* stream) {
    int rc;
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz))) return rc;
    const int eb = elem_align(storage);
    if ((rc = check_ptr(phi, eb, "phi")) || (rc = check_ptr(out, 8, "out")) ||
        (rc = check_ptr(workspace, 8, "workspace")))
        return rc;
    if (pi && (rc = check_ptr(pi, eb, "pi"))) return rc;
    // (nx, ny, 1) is the same C-order memory as (1, nx, ny): walk rows of length ny
    if (nz == 1) {
        nz = ny;
        ny = nx;
        nx = 1;
    }
    const int64_t need = obs_workspace_bytes((int)nx, (int)ny, (int)nz);
    if (workspace_bytes < need)
        return fail(TIPT_ERR_ARG, "workspace of %lld bytes is smaller than the %lld needed",
                    (long long)workspace_bytes, (long long)need);
    return launch_observables(storage, phi, pi, (int)nx, (int)ny, (int)nz, 0, (int)nx,
                              (double)(nx * ny * nz), dx, inv_a2, lam, mphi, mu, thr, out,
                              static_cast<double*>(workspace), (cudaStream_t)stream);
}

extern "C" int tipt_observables_slab(int storage, const void* phi, const void* pi,
                                     int64_t nx_local, int64_t ny, int64_t nz,
                                     int64_t n_global_sites, double dx, double inv_a2, double lam,
                                     double mphi, double mu, double thr, double* out,
                                     void* workspace, int64_t workspace_bytes, void* stream) {
    int rc;
    if (nx_local < 1 || nz < 2)
        return fail(TIPT_ERR_ARG, "slab needs nx_local >= 1 and nz >= 2");
    const int64_t n0 = nx_local + 2;
    if ((rc = check_storage(storage)) || (rc = check_dims(n0, ny, nz))) return rc;
    if (n_global_sites < nx_local * ny * nz)
        return fail(TIPT_ERR_ARG, "n_global_sites smaller than the slab");
    const int eb = elem_align(storage);
    if ((rc = check_ptr(phi, eb, "phi")) || (rc = check_ptr(out, 8, "out")) ||
        (rc = check_ptr(workspace, 8, "workspace")))
        return rc;
    if (pi && (rc = check_ptr(pi, eb, "pi"))) return rc;
    const int64_t need = obs_workspace_bytes((int)n0, (int)ny, (int)nz);
    if (workspace_bytes < need)
        return fail(TIPT_ERR_ARG, "workspace of %lld bytes is smaller than the %lld needed",
                    (long long)workspace_bytes, (long long)need);
    return launch_observables(storage, phi, pi, (int)n0, (int)ny, (int)nz, 1, (int)nx_local + 1,
                              (double)n_global_sites, dx, inv_a2, lam, mphi, mu, thr, out,
                              static_cast<double*>(workspace), (cudaStream_t)stream);
}
