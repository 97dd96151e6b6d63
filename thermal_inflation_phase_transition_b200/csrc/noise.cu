// Counter-based noise kernels: the hash pairs themselves (parity checks) and
// the noise-field fill that replaces the MT19937 generate_noise_field.
#include "tipt_device.cuh"
#include "tipt_internal.h"

namespace tipt {

__global__ void hash_pairs_kernel(const uint64_t* __restrict__ keys, int64_t n, double* u1,
                                  double* u2, double* z) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        double a, b;
        hash_pair(keys[q], a, b);
        if (u1) u1[q] = a;
        if (u2) u2[q] = b;
        if (z) z[q] = bm_radius(a) * cos(kTwoPiLit * b);
    }
}

template <typename OT>
__global__ void noise_fill_kernel(OT* __restrict__ out, int64_t N, double scale, uint64_t step,
                                  uint64_t mul, uint64_t seed, int component) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double u1, u2;
        hash_pair(noise_key((uint64_t)s, step, mul, seed), u1, u2);
        double r = bm_radius(u1);
        double v = component ? r * sin(kTwoPiLit * u2) : r * cos(kTwoPiLit * u2);
        out[s] = (OT)(scale * v);
    }
}

static unsigned grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)num_sms() * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

int launch_hash_pairs(const uint64_t* keys, int64_t n, double* u1, double* u2, double* z,
                      cudaStream_t st) {
    if (n == 0) return TIPT_OK;
    hash_pairs_kernel<<<grid_for(n, 256), 256, 0, st>>>(keys, n, u1, u2, z);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "hash_pairs launch");
}

int launch_noise_fill(int storage, void* out, int64_t N, double scale, uint64_t step,
                      uint64_t mul, uint64_t seed, int component, cudaStream_t st) {
    if (N == 0) return TIPT_OK;
    if (storage == TIPT_F64)
        noise_fill_kernel<double><<<grid_for(N, 256), 256, 0, st>>>(
            static_cast<double*>(out), N, scale, step, mul, seed, component);
    else
        noise_fill_kernel<float><<<grid_for(N, 256), 256, 0, st>>>(
            static_cast<float*>(out), N, scale, step, mul, seed, component);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "noise_fill launch");
}

}  // namespace tipt
