// Plaquette winding numbers: compute_winding_number (C:2683-2744,
// tools/winding.py:15-64) and the string count of C:4661.
//
// The reference sums atan2(sin d, cos d) over the four edges of each
// plaquette and divides by 2 pi.  atan2(sin d, cos d) equals d - 2 pi m with
// m = +1 for d > pi, -1 for d < -pi and 0 otherwise (d itself is a difference
// of two atan2 values in [-pi, pi], so |d| < 2 pi), and the four raw
// differences telescope to zero.  The plaquette winding is therefore the
// integer -(m1 + m2 + m3 + m4), computed here exactly from the four wrap
// decisions instead of from the rounded floating sum.
#include "tipt_device.cuh"
#include "tipt_internal.h"

namespace tipt {

constexpr double kPiD = 3.141592653589793;  // the double nearest pi (numpy's np.pi)

__device__ __forceinline__ int wrap_count(double d) { return d > kPiD ? 1 : (d < -kPiD ? -1 : 0); }

// Site value in FP64; F32C is planar (hi plane, then lo plane N sites later).
template <int S>
__device__ __forceinline__ double load_field(const void* p, int64_t s, int64_t N) {
    if constexpr (S == TIPT_F64) return __ldg(static_cast<const double*>(p) + s);
    else if constexpr (S == TIPT_F32) return (double)__ldg(static_cast<const float*>(p) + s);
    else {
        const float* f = static_cast<const float*>(p);
        return (double)__ldg(f + s) + (double)__ldg(f + N + s);
    }
}

struct WindParams {
    const void* phi1;
    const void* phi2;
    int n0, n1, n2;
    float* w_site;
    int8_t* w3;
    uint32_t* pierced;
    int64_t cap;
    unsigned long long* counts;  // [5]
};

// Tiled kernel.  A block takes a tile of TI x TJ x TK sites (k contiguous) and
// its forward halo (one more plane, row and column, periodic): the phase of
// every halo-region site is computed once (FP64 atan2 of the FP64 field
// values, as the reference computes it on FP64 casts, C:4627-4629) into shared
// memory, then the wrap count of each forward edge,
//   e_i(s) = wrap(theta(s + i) - theta(s)),  e_j, e_k alike,
// and every plaquette is a signed sum of four edge counts: the reference's
// atan2(sin d, cos d) over an edge traversed backwards is the wrap of -d, and
// IEEE subtraction gives (a - b) = -(b - a) exactly, so wrap(-d) = -wrap(d):
//   XY(s) = -(e_i(s) + e_j(s + i) - e_i(s + j) - e_j(s)),  XZ, YZ alike.
// One atan2 per region site instead of seven per site, and 3 FP64
// differences per site instead of 12; the decisions are those of the
// reference's per-plaquette differences bit for bit.
template <int TK>
struct WindTile {
    static constexpr int TJ = TK == 32 ? 8 : (TK == 8 ? 16 : 64);
    static constexpr int TI = TK == 32 ? 8 : (TK == 8 ? 16 : 32);
    static constexpr int RI = TI + 1, RJ = TJ + 1, RK = TK + 1;
    static constexpr int REGION = RI * RJ * RK;
    static constexpr int INTERIOR = TI * TJ * TK;
};

template <int S, int TK>
__global__ void __launch_bounds__(256) winding_tiled_kernel(WindParams p) {
    using W = WindTile<TK>;
    __shared__ double s_th[W::REGION];
    __shared__ int8_t s_e[3][W::REGION];
    const int64_t n12 = (int64_t)p.n1 * p.n2;
    const int64_t N = (int64_t)p.n0 * n12;
    const int nti = (p.n0 + W::TI - 1) / W::TI, ntj = (p.n1 + W::TJ - 1) / W::TJ,
              ntk = (p.n2 + TK - 1) / TK;
    const int64_t tiles = (int64_t)nti * ntj * ntk;
    const unsigned lane = threadIdx.x & 31;
    unsigned long long c_xy = 0, c_xz = 0, c_yz = 0, c_str = 0;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int tk = (int)(tile % ntk);
        const int64_t tr = tile / ntk;
        const int tj = (int)(tr % ntj), ti = (int)(tr / ntj);
        const int i0 = ti * W::TI, j0 = tj * W::TJ, k0 = tk * TK;
        // phases of the region (coordinates taken modulo the lattice)
        for (int q = threadIdx.x; q < W::REGION; q += blockDim.x) {
            const int c = q % W::RK, rr = q / W::RK;
            const int b = rr % W::RJ, a = rr / W::RJ;
            const int i = (i0 + a) % p.n0, j = (j0 + b) % p.n1, k = (k0 + c) % p.n2;
            const int64_t sq = (int64_t)i * n12 + (int64_t)j * p.n2 + k;
            s_th[q] = atan2(load_field<S>(p.phi2, sq, N), load_field<S>(p.phi1, sq, N));
        }
        __syncthreads();
        // forward-edge wrap counts (the far faces are never read)
        for (int q = threadIdx.x; q < W::REGION; q += blockDim.x) {
            const int c = q % W::RK, rr = q / W::RK;
            const int b = rr % W::RJ, a = rr / W::RJ;
            const double t = s_th[q];
            s_e[0][q] = (int8_t)(a < W::TI ? wrap_count(s_th[q + W::RJ * W::RK] - t) : 0);
            s_e[1][q] = (int8_t)(b < W::TJ ? wrap_count(s_th[q + W::RK] - t) : 0);
            s_e[2][q] = (int8_t)(c < TK ? wrap_count(s_th[q + 1] - t) : 0);
        }
        __syncthreads();
        // plaquettes: warp-uniform trip count (the ballots need full warps)
        for (int q0 = threadIdx.x & ~31; q0 < W::INTERIOR; q0 += blockDim.x) {
            const int q = q0 + (int)lane;
            const int c = q % TK, rr = q / TK;
            const int b = rr % W::TJ, a = rr / W::TJ;
            const int i = i0 + a, j = j0 + b, k = k0 + c;
            const bool live = i < p.n0 && j < p.n1 && k < p.n2;
            int wxy = 0, wxz = 0, wyz = 0;
            int64_t s = 0;
            if (live) {
                const int r0 = (a * W::RJ + b) * W::RK + c;
                const int ri = r0 + W::RJ * W::RK, rj = r0 + W::RK, rk = r0 + 1;
                wxy = -(s_e[0][r0] + s_e[1][ri] - s_e[0][rj] - s_e[1][r0]);
                wxz = -(s_e[0][r0] + s_e[2][ri] - s_e[0][rk] - s_e[2][r0]);
                wyz = -(s_e[1][r0] + s_e[2][rj] - s_e[1][rk] - s_e[2][r0]);
                s = (int64_t)i * n12 + (int64_t)j * p.n2 + k;
                const int w = wxy + wxz + wyz;
                if (p.w_site) p.w_site[s] = (float)w;
                if (p.w3) {
                    p.w3[s] = (int8_t)wxy;
                    p.w3[N + s] = (int8_t)wxz;
                    p.w3[2 * N + s] = (int8_t)wyz;
                }
                c_xy += wxy != 0;
                c_xz += wxz != 0;
                c_yz += wyz != 0;
                c_str += w != 0;  // |w| > 0.5 for integer w
            }
            if (p.pierced) {
                // warp-ballot compaction: one atomic per warp and orientation
                const int wo[3] = {wxy, wxz, wyz};
#pragma unroll
                for (int o = 0; o < 3; ++o) {
                    const unsigned m = __ballot_sync(0xffffffffu, live && wo[o] != 0);
                    if (m == 0) continue;
                    unsigned long long b0 = 0;
                    if (lane == 0) b0 = atomicAdd(&p.counts[4], (unsigned long long)__popc(m));
                    b0 = __shfl_sync(0xffffffffu, b0, 0);
                    if (live && wo[o] != 0) {
                        const unsigned long long slot = b0 + __popc(m & ((1u << lane) - 1u));
                        if ((int64_t)slot < p.cap) p.pierced[slot] = (uint32_t)(s * 3 + o);
                    }
                }
            }
        }
        __syncthreads();  // the region buffers are refilled by the next tile
    }
    // warp totals -> one atomic per warp and counter
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        c_xy += __shfl_down_sync(0xffffffffu, c_xy, off);
        c_xz += __shfl_down_sync(0xffffffffu, c_xz, off);
        c_yz += __shfl_down_sync(0xffffffffu, c_yz, off);
        c_str += __shfl_down_sync(0xffffffffu, c_str, off);
    }
    if (lane == 0) {
        if (c_xy) atomicAdd(&p.counts[0], c_xy);
        if (c_xz) atomicAdd(&p.counts[1], c_xz);
        if (c_yz) atomicAdd(&p.counts[2], c_yz);
        if (c_str) atomicAdd(&p.counts[3], c_str);
    }
}

// counts[4] collects the total number of pierced plaquettes found by the
// ballots; clamp it to the list capacity afterwards.
__global__ void winding_clamp_kernel(unsigned long long* counts, int64_t cap) {
    if (counts[4] > (unsigned long long)cap) counts[4] = (unsigned long long)cap;
}

}  // namespace tipt

using namespace tipt;

extern "C" int tipt_compute_winding_number(int storage, const void* phi1, const void* phi2,
                                           int64_t nx, int64_t ny, int64_t nz, float* w_site,
                                           int8_t* w3, uint32_t* pierced, int64_t pierced_cap,
                                           int64_t* counts, void* stream) {
    int rc;
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz))) return rc;
    const int eb = elem_align(storage);
    if ((rc = check_ptr(phi1, eb, "phi1")) || (rc = check_ptr(phi2, eb, "phi2")) ||
        (rc = check_ptr(counts, 8, "counts")))
        return rc;
    if (pierced && pierced_cap < 0) return fail(TIPT_ERR_ARG, "pierced_cap < 0");
    if (nx * ny * nz * 3 > 0xFFFFFFFFll && pierced)
        return fail(TIPT_ERR_UNSUPPORTED, "pierced list entries are 32-bit (N*3 < 2^32)");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(counts, 0, 5 * sizeof(int64_t), st);
    if (e != cudaSuccess) return fail_cuda(e, "winding counts memset");
    WindParams p;
    p.phi1 = phi1;
    p.phi2 = phi2;
    p.n0 = (int)nx;
    p.n1 = (int)ny;
    p.n2 = (int)nz;
    p.w_site = w_site;
    p.w3 = w3;
    p.pierced = pierced;
    p.cap = pierced ? pierced_cap : 0;
    p.counts = reinterpret_cast<unsigned long long*>(counts);
    // tile shape by the contiguous extent: 8 x 8 x 32, 16 x 16 x 8 or 32 x 64 x 1
    const int tk = nz >= 24 ? 32 : (nz >= 6 ? 8 : 1);
    const int64_t cap_blocks = (int64_t)num_sms() * 8;
    auto grid = [&](int ti, int tj, int tkk) {
        const int64_t nb = ((nx + ti - 1) / ti) * ((ny + tj - 1) / tj) * ((nz + tkk - 1) / tkk);
        return (unsigned)(nb < cap_blocks ? nb : cap_blocks);
    };
    if (tk == 32) {
        const unsigned nb = grid(WindTile<32>::TI, WindTile<32>::TJ, 32);
        if (storage == TIPT_F64) winding_tiled_kernel<TIPT_F64, 32><<<nb, 256, 0, st>>>(p);
        else if (storage == TIPT_F32) winding_tiled_kernel<TIPT_F32, 32><<<nb, 256, 0, st>>>(p);
        else winding_tiled_kernel<TIPT_F32C, 32><<<nb, 256, 0, st>>>(p);
    } else if (tk == 8) {
        const unsigned nb = grid(WindTile<8>::TI, WindTile<8>::TJ, 8);
        if (storage == TIPT_F64) winding_tiled_kernel<TIPT_F64, 8><<<nb, 256, 0, st>>>(p);
        else if (storage == TIPT_F32) winding_tiled_kernel<TIPT_F32, 8><<<nb, 256, 0, st>>>(p);
        else winding_tiled_kernel<TIPT_F32C, 8><<<nb, 256, 0, st>>>(p);
    } else {
        const unsigned nb = grid(WindTile<1>::TI, WindTile<1>::TJ, 1);
        if (storage == TIPT_F64) winding_tiled_kernel<TIPT_F64, 1><<<nb, 256, 0, st>>>(p);
        else if (storage == TIPT_F32) winding_tiled_kernel<TIPT_F32, 1><<<nb, 256, 0, st>>>(p);
        else winding_tiled_kernel<TIPT_F32C, 1><<<nb, 256, 0, st>>>(p);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "winding launch");
    if (pierced) {
        winding_clamp_kernel<<<1, 1, 0, st>>>(p.counts, p.cap);
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail_cuda(e, "winding clamp launch");
    }
    return TIPT_OK;
}
