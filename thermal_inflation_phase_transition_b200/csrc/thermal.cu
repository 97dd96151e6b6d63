// Thermal one-loop V' of the physics-default potential (R:432-496, R:755-849,
// R:1415-1485): FP64 quadrature of dJ_B/du and dJ_F/du on a uniform grid of
// u = m/T, the lattice counterterm's soft-mode subtraction, and the V'
// assembly (Vprime_field / Vprime_scalar) from cubic-spline coefficients,
// per site or over a (phi, T) grid for the stepper's 2-D V' table.
//
//   dJ_B(u) = int_0^100 y^2 u / (E (e^E - 1)) dy,  dJ_F(u) = int_0^100 y^2 u / (E (e^E + 1)) dy,
//   E = sqrt(y^2 + u^2)  (the integrals of cosmoTransitions' finiteT.dJb_exact /
//   dJf_exact, restated in potential/flatonPotential.py _dJb_exact/_dJf_exact);
//   soft part (R:461-490): (1 / 2 pi^2) int_0^{x_cut} x^2 u / (z (e^z -/+ 1)) dx,
//   z = sqrt(x^2 + u^2), integrand 0 where z > 50.
// Quadrature: composite 16-point Gauss-Legendre on equal panels (nodes and
// weights from the host), one block per grid point, fixed-order sums.
#include "tipt_device.cuh"
#include "tipt_internal.h"

namespace tipt {

constexpr int kGL = 16;
constexpr int kPanels = 2048;

struct GLRule {
    double x[kGL], w[kGL];  // nodes and weights on [-1, 1]
};

__device__ __forceinline__ double dj_integrand(double y, double u, int fermion) {
    const double E = sqrt(y * y + u * u);
    const double den = fermion ? (exp(E) + 1.0) : expm1(E);
    return y * y * u / (E * den);
}

__device__ __forceinline__ double soft_integrand(double x, double u, int fermion) {
    const double z = sqrt(x * x + u * u);
    if (z > 50.0) return 0.0;
    const double den = fermion ? (exp(z) + 1.0) : expm1(z);
    return x * x * u / (z * den);
}

// composite Gauss-Legendre over [0, b]: panel sums in a fixed per-thread order,
// then a fixed tree over the block
template <bool SOFT>
__device__ double panel_integral(const GLRule& gl, double b, double u, int fermion, double* s_red) {
    const double hp = b / kPanels;
    double acc = 0.0;
    for (int q = threadIdx.x; q < kPanels; q += blockDim.x) {
        const double a0 = q * hp, half = 0.5 * hp;
        double ps = 0.0;
#pragma unroll
        for (int n = 0; n < kGL; ++n) {
            const double y = a0 + half * (1.0 + gl.x[n]);
            ps += gl.w[n] * (SOFT ? soft_integrand(y, u, fermion) : dj_integrand(y, u, fermion));
        }
        acc += half * ps;
    }
    s_red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s_red[threadIdx.x] += s_red[threadIdx.x + w];
        __syncthreads();
    }
    const double r = s_red[0];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(256) dj_kernel(GLRule gl, const double* u, int fermion,
                                                 double x_cut, double* out) {
    __shared__ double s_red[256];
    const double uu = u[blockIdx.x];
    double v = uu == 0.0 ? 0.0 : panel_integral<false>(gl, 100.0, uu, fermion, s_red);
    if (x_cut >= 1e-10 && uu >= 1e-30) {
        const double soft = panel_integral<true>(gl, x_cut, uu, fermion, s_red);
        v -= soft / (2.0 * 3.141592653589793 * 3.141592653589793);
    }
    if (threadIdx.x == 0) out[blockIdx.x] = v;
}

// ---------------------------------------------------------------- V' ----
// R:1415 cubic_eval_uniform: segment of x (trunc, clamped to [0, nseg-1]),
// Horner in dx = x - x_i with coefficients for dx^3, dx^2, dx, 1.
__device__ __forceinline__ double cubic_eval(const double* c, int nseg, double x_min, double h,
                                             double x) {
    int i = (int)((x - x_min) / h);
    i = i < 0 ? 0 : (i >= nseg ? nseg - 1 : i);
    const double dx = x - (x_min + i * h);
    return ((c[i] * dx + c[nseg + i]) * dx + c[2 * nseg + i]) * dx + c[3 * nseg + i];
}

// R:1435-1485 Vprime_field at one site.
__device__ double thermal_vprime(const tipt_thermal& t, double ph, double T) {
    const double T2 = T * T;
    const double pref = T2 * T2 / (2.0 * 3.141592653589793 * 3.141592653589793);
    const double gb2 = t.boson_coupling * t.boson_coupling;
    const double gg2 = t.boson_gauge_coupling * t.boson_gauge_coupling;
    const double gf2 = t.fermion_coupling * t.fermion_coupling;
    const double gfg2 = t.fermion_gauge_coupling * t.fermion_gauge_coupling;
    const double coef_b_T = 0.25 * gb2 + (2.0 / 3.0) * gg2;
    double dV = t.lam * ph * ph * ph - t.mphi * t.mphi * ph;
    const double xb_sq = t.boson_mass_sq + 0.5 * gb2 * ph * ph + coef_b_T * T2;
    const double xb = xb_sq > 0.0 ? sqrt(xb_sq) / T : 0.0;
    const double xf_sq = 0.5 * gf2 * ph * ph + (1.0 / 6.0) * gfg2 * T2;
    const double xf = xf_sq > 0.0 ? sqrt(xf_sq) / T : 0.0;
    const double hi = t.x_min + t.h * t.nseg;
    const double xbc = xb < t.x_min ? t.x_min : (xb > hi ? hi - 1e-12 : xb);
    const double xfc = xf < t.x_min ? t.x_min : (xf > hi ? hi - 1e-12 : xf);
    const double djb = cubic_eval(t.spline, t.nseg, t.x_min, t.h, xbc);
    const double djf = cubic_eval(t.spline + 4 * t.nseg, t.nseg, t.x_min, t.h, xfc);
    const double dxb = 0.5 * gb2 * ph / (T2 * fmax(xb, 1e-20));
    const double dxf = 0.5 * gf2 * ph / (T2 * fmax(xf, 1e-20));
    return dV + pref * (t.coeff_b * djb * dxb + t.coeff_f * djf * dxf);
}

template <int S>
__global__ void thermal_field_kernel(const void* phi, double T, tipt_thermal t, double* out,
                                     int64_t N) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double ph;
        if constexpr (S == TIPT_F64) ph = static_cast<const double*>(phi)[s];
        else if constexpr (S == TIPT_F32) ph = (double)static_cast<const float*>(phi)[s];
        else {
            const float* f = static_cast<const float*>(phi);
            ph = (double)f[s] + (double)f[N + s];
        }
        out[s] = thermal_vprime(t, ph, T);
    }
}

// table[j][i] = V'(phi_i, T_j), phi_i the numpy.linspace(phi_lo, phi_hi, nphi) grid
__global__ void thermal_table_kernel(double phi_lo, double phi_hi, int nphi, const double* Ts,
                                     int nT, tipt_thermal t, double* out) {
    const double step = (phi_hi - phi_lo) / (nphi - 1);
    const int64_t total = (int64_t)nphi * nT;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(q / nphi), i = (int)(q - (int64_t)j * nphi);
        const double ph = i == nphi - 1 ? phi_hi : phi_lo + i * step;
        out[q] = thermal_vprime(t, ph, Ts[j]);
    }
}

static int check_thermal(const tipt_thermal* t) {
    if (!t) return fail(TIPT_ERR_ARG, "thermal parameters are NULL");
    if (t->nseg < 1 || !(t->h > 0.0)) return fail(TIPT_ERR_ARG, "bad spline grid");
    return check_ptr(t->spline, 8, "spline");
}

}  // namespace tipt

using namespace tipt;

extern "C" int tipt_thermal_dj(int fermion, const double* u, int32_t n, const double* gl_nodes,
                               const double* gl_weights, double x_cut, double* out, void* stream) {
    int rc;
    if (n < 1) return fail(TIPT_ERR_ARG, "n must be >= 1");
    if ((rc = check_ptr(u, 8, "u")) || (rc = check_ptr(out, 8, "out"))) return rc;
    if (!gl_nodes || !gl_weights) return fail(TIPT_ERR_ARG, "Gauss-Legendre rule is NULL");
    GLRule gl;
    for (int q = 0; q < kGL; ++q) {
        gl.x[q] = gl_nodes[q];  // host arrays of 16 nodes / weights on [-1, 1]
        gl.w[q] = gl_weights[q];
    }
    dj_kernel<<<n, 256, 0, (cudaStream_t)stream>>>(gl, u, fermion ? 1 : 0, x_cut, out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "dJ quadrature launch");
}

extern "C" int tipt_thermal_vprime_field(int storage, const void* phi, double T,
                                         const tipt_thermal* tp, double* out, int64_t nx,
                                         int64_t ny, int64_t nz, void* stream) {
    int rc;
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz)) ||
        (rc = check_ptr(phi, elem_align(storage), "phi")) || (rc = check_ptr(out, 8, "out")) ||
        (rc = check_thermal(tp)))
        return rc;
    if (!(T > 0.0)) return fail(TIPT_ERR_ARG, "T must be > 0");
    const int64_t N = nx * ny * nz;
    int64_t blocks = (N + 255) / 256;
    if (blocks > (int64_t)num_sms() * 16) blocks = (int64_t)num_sms() * 16;
    cudaStream_t st = (cudaStream_t)stream;
    switch (storage) {
        case TIPT_F64: thermal_field_kernel<TIPT_F64><<<(unsigned)blocks, 256, 0, st>>>(phi, T, *tp, out, N); break;
        case TIPT_F32: thermal_field_kernel<TIPT_F32><<<(unsigned)blocks, 256, 0, st>>>(phi, T, *tp, out, N); break;
        default: thermal_field_kernel<TIPT_F32C><<<(unsigned)blocks, 256, 0, st>>>(phi, T, *tp, out, N); break;
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "thermal V' launch");
}

// C:1452-1530 Vprime_field of the complex field at one site: the radial V' of
// Vprime_field at rho_safe = max(rho, 1e-30), projected as V' phi_a / rho_safe,
// plus the Z_N term (C:1519-1527).
template <int S>
__global__ void thermal_field_complex_kernel(const void* phi1, const void* phi2, double T,
                                             tipt_thermal t, tipt_complex_terms ct, double* out1,
                                             double* out2, int64_t N) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double p1, p2;
        if constexpr (S == TIPT_F64) {
            p1 = static_cast<const double*>(phi1)[s];
            p2 = static_cast<const double*>(phi2)[s];
        } else if constexpr (S == TIPT_F32) {
            p1 = (double)static_cast<const float*>(phi1)[s];
            p2 = (double)static_cast<const float*>(phi2)[s];
        } else {
            const float* a = static_cast<const float*>(phi1);
            const float* b = static_cast<const float*>(phi2);
            p1 = (double)a[s] + (double)a[N + s];
            p2 = (double)b[s] + (double)b[N + s];
        }
        const double rho = sqrt(p1 * p1 + p2 * p2);
        const double rho_safe = rho > 1e-30 ? rho : 1e-30;
        const double inv_rho = 1.0 / rho_safe;
        const double dv = thermal_vprime(t, rho_safe, T);
        double d1 = dv * p1 * inv_rho, d2 = dv * p2 * inv_rho;
        if (ct.zn_active > 0.5 && ct.zn_n > 0.5 && rho > 1e-20) {
            const double sn = sin(ct.zn_n * atan2(p2, p1));
            const double ir2 = inv_rho * inv_rho;
            d1 += -ct.zn_n * ct.zn_dv * sn * p2 * ir2;
            d2 += ct.zn_n * ct.zn_dv * sn * p1 * ir2;
        }
        out1[s] = d1;
        out2[s] = d2;
    }
}

extern "C" int tipt_thermal_vprime_field_complex(int storage, const void* phi1, const void* phi2,
                                                 double T, const tipt_thermal* tp,
                                                 const tipt_complex_terms* ct, double* out1,
                                                 double* out2, int64_t nx, int64_t ny, int64_t nz,
                                                 void* stream) {
    int rc;
    const int al = elem_align(storage);
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz)) ||
        (rc = check_ptr(phi1, al, "phi1")) || (rc = check_ptr(phi2, al, "phi2")) ||
        (rc = check_ptr(out1, 8, "out1")) || (rc = check_ptr(out2, 8, "out2")) ||
        (rc = check_thermal(tp)))
        return rc;
    if (!(T > 0.0)) return fail(TIPT_ERR_ARG, "T must be > 0");
    tipt_complex_terms terms = {0.0, 0.0, 0.0, 0.0};
    if (ct) terms = *ct;
    const int64_t N = nx * ny * nz;
    int64_t blocks = (N + 255) / 256;
    if (blocks > (int64_t)num_sms() * 16) blocks = (int64_t)num_sms() * 16;
    cudaStream_t st = (cudaStream_t)stream;
    switch (storage) {
        case TIPT_F64: thermal_field_complex_kernel<TIPT_F64><<<(unsigned)blocks, 256, 0, st>>>(phi1, phi2, T, *tp, terms, out1, out2, N); break;
        case TIPT_F32: thermal_field_complex_kernel<TIPT_F32><<<(unsigned)blocks, 256, 0, st>>>(phi1, phi2, T, *tp, terms, out1, out2, N); break;
        default: thermal_field_complex_kernel<TIPT_F32C><<<(unsigned)blocks, 256, 0, st>>>(phi1, phi2, T, *tp, terms, out1, out2, N); break;
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "complex thermal V' launch");
}

extern "C" int tipt_thermal_vprime_table(double phi_lo, double phi_hi, int32_t nphi,
                                         const double* Ts, int32_t nT, const tipt_thermal* tp,
                                         double* out, void* stream) {
    int rc;
    if (nphi < 2 || nT < 1) return fail(TIPT_ERR_ARG, "need nphi >= 2 and nT >= 1");
    if (!(phi_hi > phi_lo)) return fail(TIPT_ERR_ARG, "phi_hi must exceed phi_lo");
    if ((rc = check_ptr(Ts, 8, "T")) || (rc = check_ptr(out, 8, "out")) || (rc = check_thermal(tp)))
        return rc;
    const int64_t total = (int64_t)nphi * nT;
    int64_t blocks = (total + 255) / 256;
    if (blocks > (int64_t)num_sms() * 16) blocks = (int64_t)num_sms() * 16;
    thermal_table_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(phi_lo, phi_hi, nphi,
                                                                            Ts, nT, *tp, out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "thermal table launch");
}
