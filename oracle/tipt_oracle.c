/*
 * tipt_oracle.c -- CPU restatement of the reference lattice Langevin stepper.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it; the product
 * (the CUDA library and its Python host) never links, loads or calls it.
 *
 * Every routine restates one reference function, cited as
 *   R:  simulation/latticeSimeRescale_numba.py
 *   C:  simulation/latticeSimComplex_numba.py
 * and follows its order of floating-point operations (no FMA contraction: the
 * recipe builds with -ffp-contract=off) so that FP64 results agree with the
 * reference kernels to rounding.  Features the reference lacks but the CUDA
 * path adds (a noise seed, a 2-D (phi,T) table, the eps*Re(Phi^4) term,
 * per-orientation integer windings) are restated here from their definitions.
 *
 * Layout: C-order (nx, ny, nz) arrays, site = i*ny*nz + j*nz + k, periodic.
 * Parallelism: OpenMP over i, like the reference's nb.prange(nx).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define K_PASS2 73856093ULL
#define K_PASS4 19349669ULL
#define SEED_STRIDE 0x9E3779B97F4A7C15ULL
#define TWO_PI_LIT 6.283185307179586

/* ------------------------------------------------------------------ hash */

/* R:2322-2336 _hash_rng_pair (C:2747-2761 identical; cosmolattice_ext/
 * evolvers/stochasticrk.h:215-226 restates it).  The second mix of the
 * reference kernel is partial (no >>27 / 0x94D0.. round); the pure-Python
 * copy in tools/check_nucleation_parity.py:69-77 uses a full mix for u2 and
 * therefore does not reproduce the kernel -- the kernel is followed here. */
static inline void hash_pair(uint64_t x, double *u1, double *u2) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    x = x ^ (x >> 31);
    double a = (double)(x >> 11) * (1.0 / 9007199254740992.0);
    x = (x * 0x2545F4914F6CDD1DULL) ^ 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = x ^ (x >> 31);
    double b = (double)(x >> 11) * (1.0 / 9007199254740992.0);
    if (a < 1e-12) a = 1e-12;
    *u1 = a;
    *u2 = b;
}

/* R:2511-2520 / R:2636-2645: key = uint64(site*mul) ^ uint64(step).
 * Extension (no reference counterpart): + seed * 0x9E3779B97F4A7C15 (mod 2^64),
 * which is exactly the reference key at seed = 0. */
static inline uint64_t noise_key(int64_t site, uint64_t step, uint64_t mul, uint64_t seed) {
    return (((uint64_t)site * mul) ^ step) + seed * SEED_STRIDE;
}

/* R:2519-2521 Box-Muller (cos branch); C:2965-2970 adds the sin branch. */
static inline double bm_cos(double u1, double u2) {
    return sqrt(-2.0 * log(u1)) * cos(TWO_PI_LIT * u2);
}
static inline double bm_sin(double u1, double u2) {
    return sqrt(-2.0 * log(u1)) * sin(TWO_PI_LIT * u2);
}

void orc_hash_pair(const uint64_t *seeds, int64_t n, double *u1, double *u2, double *z) {
    for (int64_t s = 0; s < n; ++s) {
        double a, b;
        hash_pair(seeds[s], &a, &b);
        u1[s] = a;
        u2[s] = b;
        if (z) z[s] = bm_cos(a, b);
    }
}

uint64_t orc_noise_key(int64_t site, uint64_t step, uint64_t mul, uint64_t seed) {
    return noise_key(site, step, mul, seed);
}

/* Noise field: out[site] = scale * z(site, step, mul, seed); component 0 = cos,
 * 1 = sin (the complex field's second component, C:2968-2970). */
void orc_noise_fill(double *out, int64_t nx, int64_t ny, int64_t nz, uint64_t step,
                    uint64_t mul, uint64_t seed, double scale, int component) {
    const int64_t nyz = ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nx; ++i)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t k = 0; k < nz; ++k) {
                int64_t site = i * nyz + j * nz + k;
                double u1, u2;
                hash_pair(noise_key(site, step, mul, seed), &u1, &u2);
                out[site] = scale * (component ? bm_sin(u1, u2) : bm_cos(u1, u2));
            }
}

/* ------------------------------------------------------------- V' table */

/* R:1923-1930 lookup: fidx = (x - tmin)*dinv; idx = int(fidx) (toward 0),
 * clamped to [0, n-2]; frac = fidx - idx is NOT clamped (linear
 * extrapolation outside the table). */
static inline double table_lerp(const double *t, double tmin, double dinv, int64_t last, double x) {
    double fidx = (x - tmin) * dinv;
    int64_t idx;
    if (!(fidx > 0.0)) idx = 0;               /* covers NaN and negatives */
    else if (fidx >= (double)last) idx = last;
    else idx = (int64_t)fidx;
    double frac = fidx - (double)idx;
    return t[idx] + frac * (t[idx + 1] - t[idx]);
}

/* 2-D (phi, T) table, row-major [nT][nphi].  Bilinear lookup is done as the
 * CUDA path does it: the two rows that bracket T are blended (same trunc /
 * clamp / unclamped-weight rule as above, along T) into one row, which is then
 * lerped in phi.  out_row has nphi entries. */
void orc_table_blend_row(const double *t2d, int64_t n_T, int64_t n_phi, double T_min,
                         double T_dinv, double T, double *out_row) {
    double ft = (T - T_min) * T_dinv;
    int64_t last = n_T - 2, it;
    if (!(ft > 0.0)) it = 0;
    else if (ft >= (double)last) it = last;
    else it = (int64_t)ft;
    double w = ft - (double)it;
    const double *a = t2d + it * n_phi, *b = a + n_phi;
    for (int64_t p = 0; p < n_phi; ++p) out_row[p] = a[p] + w * (b[p] - a[p]);
}

/* V' source: a uniform table (R:1923-1930) or, when tab == NULL, the
 * polynomial V'(x) = lam*x*x*x - m2*x + c2*x*x evaluated as the inline path
 * does for zero thermal couplings (R:2228: dV = lam*ph*ph*ph - mphi_sq*ph). */
typedef struct {
    const double *tab;
    double tmin, dinv;
    int64_t last;
    double lam, m2, c2;
} vsrc_t;

static inline double vprime(const vsrc_t *v, double x) {
    if (v->tab) return table_lerp(v->tab, v->tmin, v->dinv, v->last, x);
    double d = v->lam * x * x * x - v->m2 * x;
    if (v->c2 != 0.0) d += v->c2 * x * x;
    return d;
}

/* ------------------------------------------------- real field, midpoint */

/* Noise policy shared by the steppers:
 *   noise != NULL  -> the reference convention: a caller-filled array,
 *   noise == NULL and ns != 0 -> inline hash noise ns*z(site, step, mul, seed).
 */
typedef struct {
    const double *arr;
    double ns;
    uint64_t step, seed;
} noise_src;

static inline double noise_at(const noise_src *n, int64_t site, uint64_t mul) {
    if (n->arr) return n->arr[site];
    if (n->ns == 0.0) return 0.0;
    double u1, u2;
    hash_pair(noise_key(site, n->step, mul, n->seed), &u1, &u2);
    return n->ns * bm_cos(u1, u2);
}

#define NB_LOOP_BEGIN                                              \
    _Pragma("omp parallel for schedule(static)")                   \
    for (int64_t i = 0; i < nx; ++i) {                             \
        int64_t ip = i + 1 < nx ? i + 1 : 0;                       \
        int64_t im = i - 1 >= 0 ? i - 1 : nx - 1;                  \
        for (int64_t j = 0; j < ny; ++j) {                         \
            int64_t jp = j + 1 < ny ? j + 1 : 0;                   \
            int64_t jm = j - 1 >= 0 ? j - 1 : ny - 1;              \
            for (int64_t k = 0; k < nz; ++k) {                     \
                int64_t kp = k + 1 < nz ? k + 1 : 0;               \
                int64_t km = k - 1 >= 0 ? k - 1 : nz - 1;          \
                int64_t s = (i * ny + j) * nz + k;                 \
                int64_t s_ip = (ip * ny + j) * nz + k;             \
                int64_t s_im = (im * ny + j) * nz + k;             \
                int64_t s_jp = (i * ny + jp) * nz + k;             \
                int64_t s_jm = (i * ny + jm) * nz + k;             \
                int64_t s_kp = (i * ny + j) * nz + kp;             \
                int64_t s_km = (i * ny + j) * nz + km;
#define NB_LOOP_END \
    }               \
    }               \
    }

/* One FP64 midpoint half of the reference: P1 writes (phi_tmp, pi_tmp) from
 * (phi, pi); P2 reads them and advances (phi, pi) by `h2` with the noise
 * multiplied by `nfac`.  rk2_step_table (R:1875-1966) is h1 = dt/2, h2 = dt,
 * nfac = 1; each half of rk2_fused_table (R:1708-1872) is h1 = h2 = dt/2,
 * nfac = 0.5. */
static void midpoint_f64(double *phi, double *pi, double *phi_tmp, double *pi_tmp,
                         int64_t nx, int64_t ny, int64_t nz, double h1, double h2, double dx,
                         double eta_eff, double mu, double inv_a2, const vsrc_t *vs,
                         const noise_src *ns, uint64_t mul, double nfac) {
    const double inv_dx2 = 1.0 / (dx * dx);
    const double inv_mu2 = 1.0 / (mu * mu);
    /* Pass 1 (R:1903-1933) */
    NB_LOOP_BEGIN
        double ph = phi[s], pv = pi[s];
        double lap = (phi[s_ip] + phi[s_im] + phi[s_jp] + phi[s_jm] + phi[s_kp] + phi[s_km] -
                      6.0 * ph) * inv_dx2;
        double dV = vprime(vs, ph);
        double kp_ = inv_a2 * lap - eta_eff * pv - dV * inv_mu2;
        phi_tmp[s] = ph + h1 * pv;
        pi_tmp[s] = pv + h1 * kp_;
    NB_LOOP_END
    /* Pass 2 (R:1936-1966) */
    NB_LOOP_BEGIN
        double ph = phi_tmp[s], pv = pi_tmp[s];
        double lap = (phi_tmp[s_ip] + phi_tmp[s_im] + phi_tmp[s_jp] + phi_tmp[s_jm] +
                      phi_tmp[s_kp] + phi_tmp[s_km] - 6.0 * ph) * inv_dx2;
        double dV = vprime(vs, ph);
        double kp_ = inv_a2 * lap - eta_eff * pv - dV * inv_mu2;
        double nz_ = noise_at(ns, s, mul);
        phi[s] = phi[s] + h2 * pv;
        pi[s] = pi[s] + (h2 * kp_ + nfac * nz_);
    NB_LOOP_END
}

/* Mixed-precision twin for float32 storage (the reference default,
 * USE_FLOAT32=True, R:348): the six-neighbour sum is a float32 sum, the rest
 * is FP64 (python-float scalars and the FP64 table promote), stores round to
 * float32 (R:1914-1933). */
static void midpoint_f32(float *phi, float *pi, float *phi_tmp, float *pi_tmp, int64_t nx,
                         int64_t ny, int64_t nz, double h1, double h2, double dx, double eta_eff,
                         double mu, double inv_a2, const double *tab, double tmin, double dinv,
                         int64_t npts, const noise_src *ns, uint64_t mul, double nfac,
                         const float *noise32) {
    const double inv_dx2 = 1.0 / (dx * dx);
    const double inv_mu2 = 1.0 / (mu * mu);
    const int64_t last = npts - 2;
    NB_LOOP_BEGIN
        float ph = phi[s], pv = pi[s];
        float sum6 = phi[s_ip] + phi[s_im] + phi[s_jp] + phi[s_jm] + phi[s_kp] + phi[s_km];
        double lap = ((double)sum6 - 6.0 * (double)ph) * inv_dx2;
        double dV = table_lerp(tab, tmin, dinv, last, (double)ph);
        double kp_ = inv_a2 * lap - eta_eff * (double)pv - dV * inv_mu2;
        phi_tmp[s] = (float)((double)ph + h1 * (double)pv);
        pi_tmp[s] = (float)((double)pv + h1 * kp_);
    NB_LOOP_END
    NB_LOOP_BEGIN
        float ph = phi_tmp[s], pv = pi_tmp[s];
        float sum6 = phi_tmp[s_ip] + phi_tmp[s_im] + phi_tmp[s_jp] + phi_tmp[s_jm] +
                     phi_tmp[s_kp] + phi_tmp[s_km];
        double lap = ((double)sum6 - 6.0 * (double)ph) * inv_dx2;
        double dV = table_lerp(tab, tmin, dinv, last, (double)ph);
        double kp_ = inv_a2 * lap - eta_eff * (double)pv - dV * inv_mu2;
        double nz_ = noise32 ? (double)noise32[s] : noise_at(ns, s, mul);
        phi[s] = (float)((double)phi[s] + h2 * (double)pv);
        pi[s] = (float)((double)pi[s] + (h2 * kp_ + nfac * nz_));
    NB_LOOP_END
}

/* rk2_step_table (R:1875-1966), FP64 arrays.  noise: caller array (reference
 * convention) or NULL for inline hash noise ns*z(site, step, K_PASS2, seed). */
void orc_rk2_step_table_f64(double *phi, double *pi, double *phi_tmp, double *pi_tmp,
                            int64_t nx, int64_t ny, int64_t nz, double dt, double dx,
                            double eta_eff, double mu, double inv_a2, const double *tab,
                            double tmin, double dinv, int64_t npts, const double *noise,
                            double ns, uint64_t step, uint64_t seed) {
    noise_src n = {noise, ns, step, seed};
    vsrc_t v = {tab, tmin, dinv, npts - 2, 0, 0, 0};
    midpoint_f64(phi, pi, phi_tmp, pi_tmp, nx, ny, nz, 0.5 * dt, dt, dx, eta_eff, mu, inv_a2,
                 &v, &n, K_PASS2, 1.0);
}

void orc_rk2_step_table_f32(float *phi, float *pi, float *phi_tmp, float *pi_tmp, int64_t nx,
                            int64_t ny, int64_t nz, double dt, double dx, double eta_eff,
                            double mu, double inv_a2, const double *tab, double tmin,
                            double dinv, int64_t npts, const float *noise, double ns,
                            uint64_t step, uint64_t seed) {
    noise_src n = {NULL, ns, step, seed};
    midpoint_f32(phi, pi, phi_tmp, pi_tmp, nx, ny, nz, 0.5 * dt, dt, dx, eta_eff, mu, inv_a2,
                 tab, tmin, dinv, npts, &n, K_PASS2, 1.0, noise);
}

/* rk2_fused_table (R:1708-1872): two dt/2 midpoint halves at T (table a) and
 * T_mid (table b).  Array noise: 0.5*noise added in both halves (R:1806,
 * R:1872).  Hash noise (rk2_fused_single_pass, R:2511-2522, R:2636-2647):
 * 0.5*ns*z with multiplier K_PASS2 in the first half and K_PASS4 in the
 * second. */
void orc_rk2_fused_table_f64(double *phi, double *pi, double *phi_tmp, double *pi_tmp,
                             int64_t nx, int64_t ny, int64_t nz, double dt, double dx,
                             double eta_eff, double mu, double inv_a2, const double *tab_a,
                             double tmin_a, double dinv_a, int64_t npts_a, const double *tab_b,
                             double tmin_b, double dinv_b, int64_t npts_b, const double *noise,
                             double ns, uint64_t step, uint64_t seed) {
    noise_src n = {noise, ns, step, seed};
    double h = 0.5 * dt;
    vsrc_t va = {tab_a, tmin_a, dinv_a, npts_a - 2, 0, 0, 0};
    vsrc_t vb = {tab_b, tmin_b, dinv_b, npts_b - 2, 0, 0, 0};
    midpoint_f64(phi, pi, phi_tmp, pi_tmp, nx, ny, nz, h, h, dx, eta_eff, mu, inv_a2, &va, &n,
                 K_PASS2, 0.5);
    midpoint_f64(phi, pi, phi_tmp, pi_tmp, nx, ny, nz, h, h, dx, eta_eff, mu, inv_a2, &vb, &n,
                 K_PASS4, 0.5);
}

/* rk2_fused_single_pass (R:2339-2647) for zero thermal couplings: the inline
 * V' is the polynomial lam*phi^3 - mphi^2*phi at both T and T_mid, and the
 * noise is the inline hash at K_PASS2 then K_PASS4 (0.5*ns*z each). */
void orc_rk2_fused_poly_f64(double *phi, double *pi, double *phi_tmp, double *pi_tmp,
                            int64_t nx, int64_t ny, int64_t nz, double dt, double dx,
                            double eta_eff, double mu, double inv_a2, double lam, double mphi,
                            double ns, uint64_t step, uint64_t seed) {
    noise_src n = {NULL, ns, step, seed};
    double h = 0.5 * dt;
    vsrc_t v = {NULL, 0, 0, 0, lam, mphi * mphi, 0};
    midpoint_f64(phi, pi, phi_tmp, pi_tmp, nx, ny, nz, h, h, dx, eta_eff, mu, inv_a2, &v, &n,
                 K_PASS2, 0.5);
    midpoint_f64(phi, pi, phi_tmp, pi_tmp, nx, ny, nz, h, h, dx, eta_eff, mu, inv_a2, &v, &n,
                 K_PASS4, 0.5);
}

/* rk2_step_table (R:1875-1966) with the polynomial V'(x) = c1 x + c2 x^2 +
 * c3 x^3 in place of the table (the toy potential family of the batched
 * replicas: c1 = 2D(T^2-T0^2), c2 = -3ET, c3 = lam), FP64, inline hash noise
 * ns*z(site, step, K_PASS2, seed). */
void orc_rk2_step_poly_f64(double *phi, double *pi, double *phi_tmp, double *pi_tmp,
                           int64_t nx, int64_t ny, int64_t nz, double dt, double dx,
                           double eta_eff, double mu, double inv_a2, double c1, double c2,
                           double c3, double ns, uint64_t step, uint64_t seed) {
    noise_src n = {NULL, ns, step, seed};
    vsrc_t v = {NULL, 0, 0, 0, c3, -c1, c2};
    midpoint_f64(phi, pi, phi_tmp, pi_tmp, nx, ny, nz, 0.5 * dt, dt, dx, eta_eff, mu, inv_a2,
                 &v, &n, K_PASS2, 1.0);
}

void orc_rk2_fused_table_f32(float *phi, float *pi, float *phi_tmp, float *pi_tmp, int64_t nx,
                             int64_t ny, int64_t nz, double dt, double dx, double eta_eff,
                             double mu, double inv_a2, const double *tab_a, double tmin_a,
                             double dinv_a, int64_t npts_a, const double *tab_b, double tmin_b,
                             double dinv_b, int64_t npts_b, const float *noise, double ns,
                             uint64_t step, uint64_t seed) {
    noise_src n = {NULL, ns, step, seed};
    double h = 0.5 * dt;
    midpoint_f32(phi, pi, phi_tmp, pi_tmp, nx, ny, nz, h, h, dx, eta_eff, mu, inv_a2, tab_a,
                 tmin_a, dinv_a, npts_a, &n, K_PASS2, 0.5, noise);
    midpoint_f32(phi, pi, phi_tmp, pi_tmp, nx, ny, nz, h, h, dx, eta_eff, mu, inv_a2, tab_b,
                 tmin_b, dinv_b, npts_b, &n, K_PASS4, 0.5, noise);
}

/* ----------------------------------------------------------- complex */

/* Projection of the radial table force plus the symmetry-breaking terms.
 * Radial + Z_N follow C:2137-2158: rho_safe = max(rho, 1e-30);
 * dV_a = dVdrho * phi_a / rho_safe; if Z_N active: theta = atan2(p2, p1),
 * dV1 += -N dV sin(N theta) p2 / rho_safe^2, dV2 += N dV sin(N theta) p1 / rho_safe^2.
 * eps*Re(Phi^4) (no reference counterpart): dV1 += 4 eps (p1^3 - 3 p1 p2^2),
 * dV2 += 4 eps (3 p1^2 p2 - p2^3) -- the gradient of eps*(p1^4 - 6 p1^2 p2^2 + p2^4). */
typedef struct {
    double zn_n, zn_dv, zn_active, eps4;
} cplx_terms;

static inline void cplx_force(double p1, double p2, const double *tab, double tmin, double dinv,
                              int64_t last, const cplx_terms *ct, double *dV1, double *dV2) {
    double rho = sqrt(p1 * p1 + p2 * p2);
    double rho_safe = rho > 1e-30 ? rho : 1e-30;
    double dVdr = table_lerp(tab, tmin, dinv, last, rho);
    double a = dVdr * p1 / rho_safe;
    double b = dVdr * p2 / rho_safe;
    if (ct->zn_active > 0.5 && ct->zn_n > 0.5 && rho > 1e-20) {
        double th = atan2(p2, p1);
        double sn = sin(ct->zn_n * th);
        double ir2 = (1.0 / rho_safe) * (1.0 / rho_safe);
        a += -ct->zn_n * ct->zn_dv * sn * p2 * ir2;
        b += ct->zn_n * ct->zn_dv * sn * p1 * ir2;
    }
    if (ct->eps4 != 0.0) {
        a += 4.0 * ct->eps4 * (p1 * p1 * p1 - 3.0 * p1 * p2 * p2);
        b += 4.0 * ct->eps4 * (3.0 * p1 * p1 * p2 - p2 * p2 * p2);
    }
    *dV1 = a;
    *dV2 = b;
}

/* Complex rk2_step_table (C:2067-2215) in FP64.  Hash noise (no reference
 * midpoint-hash counterpart; the pair convention is C:2958-2974): one (u1,u2)
 * per site, z1 = r cos -> pi1, z2 = r sin -> pi2. */
void orc_rk2_step_table_complex_f64(double *phi1, double *phi2, double *pi1, double *pi2,
                                    double *t1, double *t2, double *tp1, double *tp2,
                                    int64_t nx, int64_t ny, int64_t nz, double dt, double dx,
                                    double eta_eff, double mu, double inv_a2, const double *tab,
                                    double tmin, double dinv, int64_t npts, double zn_n,
                                    double zn_dv, double zn_active, double eps4,
                                    const double *noise1, const double *noise2, double ns,
                                    uint64_t step, uint64_t seed) {
    const double inv_dx2 = 1.0 / (dx * dx);
    const double inv_mu2 = 1.0 / (mu * mu);
    const double half_dt = 0.5 * dt;
    const int64_t last = npts - 2;
    cplx_terms ct = {zn_n, zn_dv, zn_active, eps4};
    NB_LOOP_BEGIN
        double p1 = phi1[s], p2 = phi2[s], v1 = pi1[s], v2 = pi2[s];
        double l1 = (phi1[s_ip] + phi1[s_im] + phi1[s_jp] + phi1[s_jm] + phi1[s_kp] +
                     phi1[s_km] - 6.0 * p1) * inv_dx2;
        double l2 = (phi2[s_ip] + phi2[s_im] + phi2[s_jp] + phi2[s_jm] + phi2[s_kp] +
                     phi2[s_km] - 6.0 * p2) * inv_dx2;
        double d1, d2;
        cplx_force(p1, p2, tab, tmin, dinv, last, &ct, &d1, &d2);
        double k1 = inv_a2 * l1 - eta_eff * v1 - d1 * inv_mu2;
        double k2 = inv_a2 * l2 - eta_eff * v2 - d2 * inv_mu2;
        t1[s] = p1 + half_dt * v1;
        t2[s] = p2 + half_dt * v2;
        tp1[s] = v1 + half_dt * k1;
        tp2[s] = v2 + half_dt * k2;
    NB_LOOP_END
    NB_LOOP_BEGIN
        double p1 = t1[s], p2 = t2[s], v1 = tp1[s], v2 = tp2[s];
        double l1 = (t1[s_ip] + t1[s_im] + t1[s_jp] + t1[s_jm] + t1[s_kp] + t1[s_km] -
                     6.0 * p1) * inv_dx2;
        double l2 = (t2[s_ip] + t2[s_im] + t2[s_jp] + t2[s_jm] + t2[s_kp] + t2[s_km] -
                     6.0 * p2) * inv_dx2;
        double d1, d2;
        cplx_force(p1, p2, tab, tmin, dinv, last, &ct, &d1, &d2);
        double k1 = inv_a2 * l1 - eta_eff * v1 - d1 * inv_mu2;
        double k2 = inv_a2 * l2 - eta_eff * v2 - d2 * inv_mu2;
        double n1 = 0.0, n2 = 0.0;
        if (noise1) {
            n1 = noise1[s];
            n2 = noise2[s];
        } else if (ns != 0.0) {
            double u1, u2;
            hash_pair(noise_key(s, step, K_PASS2, seed), &u1, &u2);
            n1 = ns * bm_cos(u1, u2);
            n2 = ns * bm_sin(u1, u2);
        }
        phi1[s] = phi1[s] + dt * v1;
        phi2[s] = phi2[s] + dt * v2;
        pi1[s] = pi1[s] + (dt * k1 + n1);
        pi2[s] = pi2[s] + (dt * k2 + n2);
    NB_LOOP_END
}

/* ----------------------------------------------------------- winding */

/* compute_winding_number (C:2683-2744; tools/winding.py:26-64).  Per site the
 * XY, XZ, YZ plaquettes anchored at (i,j,k); each edge difference is wrapped
 * with atan2(sin d, cos d) and a plaquette contributes sum/(2 pi).
 * w_site (float32, like the reference's winding_buf, C:3575) is the sum over
 * the three orientations.  w3 (optional, [3][N] int8, orientation order
 * XY, XZ, YZ) holds each plaquette's rounded winding; counts[0..2] are the
 * numbers of pierced plaquettes per orientation and counts[3] the number of
 * sites with |w_site| > 0.5 (the reference string count, C:4661). */
static inline double wrapd(double d) { return atan2(sin(d), cos(d)); }

void orc_winding(const double *phi1, const double *phi2, int64_t nx, int64_t ny, int64_t nz,
                 float *w_site, int8_t *w3, int64_t *counts) {
    const int64_t N = nx * ny * nz;
    int64_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;
#pragma omp parallel for schedule(static) reduction(+ : c0, c1, c2, c3)
    for (int64_t i = 0; i < nx; ++i) {
        int64_t ip = i + 1 < nx ? i + 1 : 0;
        for (int64_t j = 0; j < ny; ++j) {
            int64_t jp = j + 1 < ny ? j + 1 : 0;
            for (int64_t k = 0; k < nz; ++k) {
                int64_t kp = k + 1 < nz ? k + 1 : 0;
#define TH(a, b, c) atan2(phi2[((a) * ny + (b)) * nz + (c)], phi1[((a) * ny + (b)) * nz + (c)])
                double th00 = TH(i, j, k), th10 = TH(ip, j, k), th11 = TH(ip, jp, k),
                       th01 = TH(i, jp, k), th1kp = TH(ip, j, kp), th0kp = TH(i, j, kp),
                       thj1kp = TH(i, jp, kp);
#undef TH
                double wxy = (wrapd(th10 - th00) + wrapd(th11 - th10) + wrapd(th01 - th11) +
                              wrapd(th00 - th01)) / (2.0 * M_PI);
                double wxz = (wrapd(th10 - th00) + wrapd(th1kp - th10) + wrapd(th0kp - th1kp) +
                              wrapd(th00 - th0kp)) / (2.0 * M_PI);
                double wyz = (wrapd(th01 - th00) + wrapd(thj1kp - th01) + wrapd(th0kp - thj1kp) +
                              wrapd(th00 - th0kp)) / (2.0 * M_PI);
                double w = 0.0;
                w += wxy;
                w += wxz;
                w += wyz;
                int64_t s = (i * ny + j) * nz + k;
                if (w_site) w_site[s] = (float)w;
                int8_t a = (int8_t)lround(wxy), b = (int8_t)lround(wxz), c = (int8_t)lround(wyz);
                if (w3) {
                    w3[s] = a;
                    w3[N + s] = b;
                    w3[2 * N + s] = c;
                }
                c0 += a != 0;
                c1 += b != 0;
                c2 += c != 0;
                c3 += fabs(w) > 0.5;
            }
        }
    }
    if (counts) {
        counts[0] = c0;
        counts[1] = c1;
        counts[2] = c2;
        counts[3] = c3;
    }
}

/* --------------------------------------------------------- observables */

/* compute_energy_densities (R:2270-2319) plus the per-step observables the
 * host loop and the post-processing read: <phi>, <phi^2>, <pi^2>,
 * fraction(phi > thr) (postprocess/plot_bubble_comparison_with_frac.py:160
 * uses |phi| > esc; the config here records phi > thr), min, max, and the
 * non-finite count of the NaN guard (R:3882-3944).
 * out[0..9] = E_kin, E_grad, E_pot, <phi>, <phi^2>, <pi^2>, frac, min, max, n_nonfinite. */
void orc_observables_f64(const double *phi, const double *pi, int64_t nx, int64_t ny, int64_t nz,
                         double dx, double inv_a2, double lam, double mphi, double mu, double thr,
                         double *out) {
    const double inv_dx2 = 1.0 / (dx * dx), inv_mu2 = 1.0 / (mu * mu), m2 = mphi * mphi;
    const int64_t n = nx * ny * nz;
    double sk = 0, sg = 0, sp = 0, s1 = 0, s2 = 0, sq = 0, mn = INFINITY, mx = -INFINITY;
    int64_t cf = 0, cn = 0;
#pragma omp parallel for schedule(static) reduction(+ : sk, sg, sp, s1, s2, sq, cf, cn) \
    reduction(min : mn) reduction(max : mx)
    for (int64_t i = 0; i < nx; ++i) {
        int64_t ip = i + 1 < nx ? i + 1 : 0;
        for (int64_t j = 0; j < ny; ++j) {
            int64_t jp = j + 1 < ny ? j + 1 : 0;
            for (int64_t k = 0; k < nz; ++k) {
                int64_t kp = k + 1 < nz ? k + 1 : 0;
                int64_t s = (i * ny + j) * nz + k;
                double ph = phi[s], pv = pi ? pi[s] : 0.0;
                sk += 0.5 * pv * pv;
                double a = phi[(ip * ny + j) * nz + k] - ph;
                double b = phi[(i * ny + jp) * nz + k] - ph;
                double c = phi[(i * ny + j) * nz + kp] - ph;
                sg += 0.5 * inv_a2 * (a * a + b * b + c * c) * inv_dx2;
                double ph2 = ph * ph;
                sp += (0.25 * lam * ph2 * ph2 - 0.5 * m2 * ph2) * inv_mu2;
                s1 += ph;
                s2 += ph2;
                sq += pv * pv;
                cf += ph > thr;
                if (!isfinite(ph) || !isfinite(pv)) cn++;
                if (ph < mn) mn = ph;
                if (ph > mx) mx = ph;
            }
        }
    }
    out[0] = sk / n;
    out[1] = sg / n;
    out[2] = sp / n;
    out[3] = s1 / n;
    out[4] = s2 / n;
    out[5] = sq / n;
    out[6] = (double)cf / n;
    out[7] = mn;
    out[8] = mx;
    out[9] = (double)cn;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
