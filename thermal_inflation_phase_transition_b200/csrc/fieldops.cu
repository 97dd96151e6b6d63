// Array helpers of the reference's un-fused stepper (rk2_step / rk2_step_fused,
// R:1488-1656): the periodic 7-point Laplacian (laplacian_periodic,
// R:1364-1385) and the uniform-grid cubic evaluation (cubic_eval_uniform,
// R:1415-1426) over an array of points.  Both are one grid-stride pass, HBM
// bound; neither is on the fused steppers' path.
#include "tipt_internal.h"

namespace tipt {

// out = (a[ip] + a[im] + a[jp] + a[jm] + a[kp] + a[km] - 6 a) / dx^2 in the
// reference's order; F32 sums the six neighbours in float32 (the reference's
// float32 arrays) and does the rest in FP64; F32C evaluates hi + lo in FP64 and
// stores the result as a {hi, lo} pair.
template <int S>
__global__ void __launch_bounds__(256) laplacian_kernel(const void* a_, void* out_, int n0, int n1,
                                                         int n2, double inv_dx2) {
    const int64_t n12 = (int64_t)n1 * n2;
    const int64_t N = (int64_t)n0 * n12;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(s % n2);
        const int64_t r = s / n2;
        const int j = (int)(r % n1);
        const int i = (int)(r / n1);
        const int64_t ip = (i + 1 < n0) ? s + n12 : s - (int64_t)(n0 - 1) * n12;
        const int64_t im = (i > 0) ? s - n12 : s + (int64_t)(n0 - 1) * n12;
        const int64_t jp = (j + 1 < n1) ? s + n2 : s - (int64_t)(n1 - 1) * n2;
        const int64_t jm = (j > 0) ? s - n2 : s + (int64_t)(n1 - 1) * n2;
        const int64_t kp = (k + 1 < n2) ? s + 1 : s - (n2 - 1);
        const int64_t km = (k > 0) ? s - 1 : s + (n2 - 1);
        if constexpr (S == TIPT_F64) {
            const double* a = static_cast<const double*>(a_);
            const double sum = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(a[ip], a[im]), a[jp]), a[jm]), a[kp]), a[km]);
            static_cast<double*>(out_)[s] = __dmul_rn(__fma_rn(-6.0, a[s], sum), inv_dx2);
        } else if constexpr (S == TIPT_F32) {
            const float* a = static_cast<const float*>(a_);
            const float sum = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(a[ip], a[im]), a[jp]), a[jm]), a[kp]), a[km]);
            static_cast<float*>(out_)[s] =
                (float)__dmul_rn(__fma_rn(-6.0, (double)a[s], (double)sum), inv_dx2);
        } else {
            const float* a = static_cast<const float*>(a_);
            auto v = [&](int64_t q) { return (double)a[q] + (double)a[N + q]; };
            const double sum = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(v(ip), v(im)), v(jp)), v(jm)), v(kp)), v(km));
            const double x = __dmul_rn(__fma_rn(-6.0, v(s), sum), inv_dx2);
            const float hi = (float)x;
            float* o = static_cast<float*>(out_);
            o[s] = hi;
            o[N + s] = (float)(x - (double)hi);
        }
    }
}

// out[n] = c0[i] dx^3 + c1[i] dx^2 + c2[i] dx + c3[i] (Horner), i = trunc((x - x_min) / h)
// clamped to [0, nseg - 1], dx = x - (x_min + i h).
__global__ void __launch_bounds__(256) cubic_kernel(const double* x, int64_t n, double x_min,
                                                     double h, int nseg, const double* c0,
                                                     const double* c1, const double* c2,
                                                     const double* c3, double* out) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
         s += (int64_t)gridDim.x * blockDim.x) {
        const double xv = x[s];
        const double t = (xv - x_min) / h;
        // trunc toward zero, clamped (NaN and out-of-int-range t take the ends)
        const int i = !(t > 0.0) ? 0 : (t >= (double)nseg ? nseg - 1 : (int)t);
        const double d = xv - (x_min + i * h);
        out[s] = ((c0[i] * d + c1[i]) * d + c2[i]) * d + c3[i];
    }
}

static unsigned grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    const int64_t cap = (int64_t)num_sms() * 8;
    return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace tipt

using namespace tipt;

extern "C" int tipt_laplacian_periodic(int storage, const void* a, void* out, int64_t nx,
                                       int64_t ny, int64_t nz, double dx, void* stream) {
    int rc;
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz))) return rc;
    const int al = elem_align(storage);
    if ((rc = check_ptr(a, al, "a")) || (rc = check_ptr(out, al, "out"))) return rc;
    const int64_t bytes = nx * ny * nz * elem_bytes(storage);
    if (overlap(a, out, bytes)) return fail(TIPT_ERR_ARG, "out overlaps a");
    if (!(dx > 0.0)) return fail(TIPT_ERR_ARG, "dx must be > 0");
    const double inv_dx2 = 1.0 / (dx * dx);
    const unsigned g = grid_for(nx * ny * nz);
    cudaStream_t st = (cudaStream_t)stream;
    switch (storage) {
        case TIPT_F64: laplacian_kernel<TIPT_F64><<<g, 256, 0, st>>>(a, out, (int)nx, (int)ny, (int)nz, inv_dx2); break;
        case TIPT_F32: laplacian_kernel<TIPT_F32><<<g, 256, 0, st>>>(a, out, (int)nx, (int)ny, (int)nz, inv_dx2); break;
        default: laplacian_kernel<TIPT_F32C><<<g, 256, 0, st>>>(a, out, (int)nx, (int)ny, (int)nz, inv_dx2); break;
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "laplacian_periodic launch");
}

extern "C" int tipt_cubic_eval_uniform(const double* x, int64_t n, double x_min, double h,
                                       int32_t nseg, const double* c0, const double* c1,
                                       const double* c2, const double* c3, double* out,
                                       void* stream) {
    int rc;
    if (n < 0) return fail(TIPT_ERR_ARG, "n must be >= 0");
    if (nseg < 1 || !(h > 0.0)) return fail(TIPT_ERR_ARG, "bad spline grid (nseg %d, h %g)", nseg, h);
    if ((rc = check_ptr(c0, 8, "c0")) || (rc = check_ptr(c1, 8, "c1")) ||
        (rc = check_ptr(c2, 8, "c2")) || (rc = check_ptr(c3, 8, "c3")))
        return rc;
    if (n == 0) return TIPT_OK;
    if ((rc = check_ptr(x, 8, "x")) || (rc = check_ptr(out, 8, "out"))) return rc;
    cubic_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(x, n, x_min, h, nseg, c0, c1, c2,
                                                                  c3, out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "cubic_eval_uniform launch");
}
