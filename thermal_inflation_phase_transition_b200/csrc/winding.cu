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

// Winding of the loop a -> b -> c -> e -> a.
__device__ __forceinline__ int plaquette(double a, double b, double c, double e) {
    return -(wrap_count(b - a) + wrap_count(c - b) + wrap_count(e - c) + wrap_count(a - e));
}

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

template <int S>
__global__ void __launch_bounds__(256) winding_kernel(WindParams p) {
    const int64_t n12 = (int64_t)p.n1 * p.n2;
    const int64_t N = (int64_t)p.n0 * n12;
    const unsigned lane = threadIdx.x & 31;
    // grid-stride loop with a warp-uniform trip count (ballots need full warps)
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t start = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    unsigned long long c_xy = 0, c_xz = 0, c_yz = 0, c_str = 0;
    for (int64_t base = start; base < N; base += stride) {
        const int64_t s = base + lane;
        const bool live = s < N;
        int wxy = 0, wxz = 0, wyz = 0;
        if (live) {
            const int k = (int)(s % p.n2);
            const int64_t r = s / p.n2;
            const int j = (int)(r % p.n1);
            const int i = (int)(r / p.n1);
            const int64_t oi = (i + 1 < p.n0) ? n12 : -(int64_t)(p.n0 - 1) * n12;
            const int64_t oj = (j + 1 < p.n1) ? (int64_t)p.n2 : -(int64_t)(p.n1 - 1) * p.n2;
            const int64_t ok = (k + 1 < p.n2) ? 1 : -(int64_t)(p.n2 - 1);
            auto th = [&](int64_t q) { return atan2(load_field<S>(p.phi2, q, N), load_field<S>(p.phi1, q, N)); };
            const double t00 = th(s), t10 = th(s + oi), t11 = th(s + oi + oj), t01 = th(s + oj);
            const double t1k = th(s + oi + ok), t0k = th(s + ok), tj1k = th(s + oj + ok);
            wxy = plaquette(t00, t10, t11, t01);   // (i,j)->(i+1,j)->(i+1,j+1)->(i,j+1)
            wxz = plaquette(t00, t10, t1k, t0k);   // (i,k)->(i+1,k)->(i+1,k+1)->(i,k+1)
            wyz = plaquette(t00, t01, tj1k, t0k);  // (j,k)->(j+1,k)->(j+1,k+1)->(j,k+1)
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
            c_str += (w > 0 ? w : -w) > 0;  // |w| > 0.5 for integer w
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
    const int64_t N = nx * ny * nz;
    int64_t blocks = (N + 255) / 256;
    const int64_t capb = (int64_t)num_sms() * 8;
    if (blocks > capb) blocks = capb;
    switch (storage) {
        case TIPT_F64: winding_kernel<TIPT_F64><<<(unsigned)blocks, 256, 0, st>>>(p); break;
        case TIPT_F32: winding_kernel<TIPT_F32><<<(unsigned)blocks, 256, 0, st>>>(p); break;
        default: winding_kernel<TIPT_F32C><<<(unsigned)blocks, 256, 0, st>>>(p); break;
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
