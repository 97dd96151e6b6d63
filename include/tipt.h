/*
 * tipt.h -- C ABI of the B200 lattice Langevin stepper (libtipt.so).
 *
 * Drop-in replacement for the numba hot path of
 *   R: simulation/latticeSimeRescale_numba.py   (real scalar field)
 *   C: simulation/latticeSimComplex_numba.py    (complex field, U(1) / Z_N)
 * Each entry point names the reference function it replaces (file:line).
 *
 * Conventions
 *  - Arrays are C-order (nx, ny, nz) device buffers, site = i*ny*nz + j*nz + k,
 *    periodic in all three directions; nz = 1 (or ny = nz = 1) gives the 2-D
 *    (1-D) lattice exactly as the reference's 7-point stencil degenerates.
 *  - State storage (`storage`): TIPT_F64 = double; TIPT_F32 = float with the
 *    reference's mixed FP32-storage / FP64-arithmetic semantics; TIPT_F32C =
 *    float2 {hi, lo} pairs per site (value hi + lo, compensated updates).
 *  - The reference updates phi, pi in place through scratch phi_tmp, pi_tmp.
 *    The fused kernels here read (phi, pi) and write (phi_out, pi_out), which
 *    must not overlap the inputs (ping-pong); the Python host restores the
 *    in-place semantics by swapping the storages.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  No entry point
 *    allocates device memory, synchronises the device or reads device memory on
 *    the host; all are capturable into CUDA graphs.  Scratch is caller-owned.
 *  - Every entry returns a tipt_status; tipt_last_error() gives the detail.
 */
#ifndef TIPT_H
#define TIPT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum {
    TIPT_OK = 0,
    TIPT_ERR_ARG = 1,         /* null pointer, bad size, aliasing, bad enum */
    TIPT_ERR_STORAGE = 2,     /* storage not supported by this entry point */
    TIPT_ERR_ALIGN = 3,       /* pointer not aligned to its element size */
    TIPT_ERR_CUDA = 4,        /* a CUDA launch or runtime call failed */
    TIPT_ERR_UNSUPPORTED = 5, /* a mode or size this build does not handle */
    TIPT_ERR_TIMEOUT = 6      /* a bounded device-side wait ran out */
} tipt_status;

enum { TIPT_F64 = 0, TIPT_F32 = 1, TIPT_F32C = 2 };

/* V' sources (R:805-849 build_vprime_table, lookup R:1923-1930). */
enum {
    TIPT_VP_TABLE = 0,   /* 1-D uniform FP64 table: table[npts] */
    TIPT_VP_TABLE2D = 1, /* 2-D FP64 table [nT][npts]; rows blended at T, then lerped in phi */
    TIPT_VP_POLY = 2,    /* V'(x) = c1 x + c2 x^2 + c3 x^3 (zero-coupling inline V', R:2228) */
    TIPT_VP_THERMAL = 3  /* the thermal one-loop V' evaluated per site at T (R:2201-2266
                            _vprime_inline): `thermal` points to its couplings and splines */
};

struct tipt_thermal;

typedef struct {
    int32_t kind;          /* TIPT_VP_* */
    int32_t npts;          /* table points along phi (>= 2) */
    const double* table;   /* device pointer */
    double tmin, dinv;     /* phi origin and 1/spacing (R:849) */
    int32_t nT;            /* 2-D: rows along T (>= 2) */
    int32_t pad_;
    double T_min, T_dinv;  /* 2-D: T origin and 1/spacing */
    double T;              /* 2-D: temperature at which rows are blended; thermal: T */
    double c1, c2, c3;     /* polynomial coefficients */
    const struct tipt_thermal* thermal; /* TIPT_VP_THERMAL: host pointer, read at the call */
} tipt_vsource;

/* Per-step scalars of the host loop (R:3674-3768): dt, dx, eta_eff, mu and
 * inv_a2 as passed to rk2_step_table; noise_scale = ns of R:3714-3718 for the
 * inline hash noise (kick ns*z per midpoint step, 0.5*ns*z per half step);
 * noise_step = the step counter n used as the hash's step (R:3742);
 * noise_seed = 0 reproduces the reference key exactly. */
typedef struct {
    double dt, dx, eta_eff, mu, inv_a2;
    double noise_scale;
    uint64_t noise_step;
    uint64_t noise_seed;
} tipt_step_params;

/* Symmetry-breaking terms of the complex field.  zn_*: the reference's
 * _ZN_PARAMS = [N, delta_V, active] (C:226-231, force C:2137-2158).
 * eps4: eps * Re(Phi^4) (no reference counterpart). */
typedef struct {
    double zn_n, zn_dv, zn_active;
    double eps4;
} tipt_complex_terms;

const char* tipt_version(void);
const char* tipt_status_string(int status);
/* Detail of the last failing call on this host thread. */
const char* tipt_last_error(void);

/* ----------------------------------------------------------------- noise */

/* _hash_rng_pair (R:2322-2336, C:2747-2761) plus the Box-Muller z of
 * R:2519-2521 for n device-resident keys.  u1, u2, z are device arrays; any
 * of them may be NULL. */
int tipt_hash_rng_pair(const uint64_t* keys, int64_t n, double* u1, double* u2, double* z,
                       void* stream);

/* Counter-based replacement of generate_noise_field (R:1348-1361), whose
 * per-thread MT19937 stream is not reproducible: out[site] = scale * z with
 * z from key(site, step, mul, seed) (R:2511-2520 seeding).  component 0 = the
 * cos branch, 1 = the sin branch (C:2968-2970).  out_storage: TIPT_F64 or
 * TIPT_F32. */
int tipt_generate_noise_field(int out_storage, void* out, int64_t nx, int64_t ny, int64_t nz,
                              double scale, uint64_t step, uint64_t mul, uint64_t seed,
                              int component, void* stream);

/* ------------------------------------------------------------ real field */

/* rk2_step_table (R:1875-1966), the reference default integrator
 * (rk2_nonfused, R:301-303): one midpoint RK2 step of size dt,
 *   k = inv_a2*lap(phi) - eta_eff*pi - V'(phi)/mu^2,
 *   phi~ = phi + dt/2 pi, pi~ = pi + dt/2 k(phi, pi),
 *   phi' = phi + dt pi~, pi' = pi + dt k(phi~, pi~) + noise,
 * fused into one launch.  noise: a device array in the state precision
 * (double for F64 and F32C, float for F32) as the reference passes it, or
 * NULL for inline hash noise noise_scale * z(site, noise_step, 73856093,
 * noise_seed). */
int tipt_rk2_step_table(int storage, const void* phi, const void* pi, void* phi_out,
                        void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                        const tipt_step_params* sp, const tipt_vsource* vp, const void* noise,
                        void* stream);

/* rk2_step_table on one x-slab of a lattice of nx_global x ny x nz sites split
 * along x across ranks (the multi-GPU form; no reference counterpart -- the
 * reference's only decomposition is CosmoLattice's MPI slabs,
 * simulation/run_cosmolattice.py:148-152).  The arrays hold nx_local + 2
 * planes: plane 0 is lattice plane i_lo - 1 and plane nx_local + 1 is lattice
 * plane i_lo + nx_local (both modulo nx_global; the ghost planes, filled by
 * the caller's halo exchange before the call), planes 1..nx_local are lattice
 * planes i_lo .. i_lo + nx_local - 1.  Computes planes 1..nx_local into
 * phi_out / pi_out (their ghost planes are not written) with the inline hash
 * noise keyed by the lattice-wide site index, so the ranks together reproduce
 * the single-lattice step bit for bit.  nz >= 2. */
int tipt_rk2_step_table_slab(int storage, const void* phi, const void* pi, void* phi_out,
                             void* pi_out, int64_t nx_local, int64_t ny, int64_t nz, int64_t i_lo,
                             int64_t nx_global, const tipt_step_params* sp,
                             const tipt_vsource* vp, void* stream);

/* tipt_rk2_step_table_slab for the array planes [plane_begin, plane_end) of
 * [1, nx_local + 1) only: the interior planes 2 .. nx_local - 1 read no ghost
 * plane and can run while the halo exchange is in flight, the two edge planes
 * after it.  No reference counterpart. */
int tipt_rk2_step_table_slab_planes(int storage, const void* phi, const void* pi, void* phi_out,
                                    void* pi_out, int64_t nx_local, int64_t ny, int64_t nz,
                                    int64_t i_lo, int64_t nx_global, int64_t plane_begin,
                                    int64_t plane_end, const tipt_step_params* sp,
                                    const tipt_vsource* vp, void* stream);

/* tipt_rk2_step_table that also reports the range of the new phi, the
 * reference loop's per-step phi.min() / phi.max() (R:3655-3660), without a
 * pass of its own: the launch folds into range[0] the minimum and into
 * range[1] the maximum of the new phi values (rounded to FP32; compensated
 * FP32: hi + lo), each as the order-preserving code c(f) = f's bits with the
 * sign bit set for f >= 0 and all bits inverted for f < 0 (decode: if the top
 * bit is set clear it, else invert), and sets range[2] = 1 if a value is NaN
 * or infinite.  The words must hold (0xFFFFFFFF, 0, 0) at the launch: the
 * launch itself resets range_next (3 words, not overlapping range) to those
 * values for the following launch, so alternating two buffers needs no
 * further launches.  No reference counterpart as one call. */
int tipt_rk2_step_table_range(int storage, const void* phi, const void* pi, void* phi_out,
                              void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                              const tipt_step_params* sp, const tipt_vsource* vp,
                              const void* noise, uint32_t* range, uint32_t* range_next,
                              void* stream);

/* rk2_step_table with the per-step scalars read on the device, for step loops
 * captured once into a CUDA graph and replayed (the reference's host loop
 * R:3619-3768 recomputes them each step on the host).  The step index is
 * s = *counter + offset; the V' 2-D table is blended at T = sched[2s], the
 * inline hash noise has amplitude sched[2s+1] and hash step
 * sp->noise_step + s.  sched is a device array of sched_len (T, ns) pairs
 * (steps beyond it reuse the last pair); counter is a device uint64 that the
 * caller advances with tipt_counter_add. */
int tipt_rk2_step_table_sched(int storage, const void* phi, const void* pi, void* phi_out,
                              void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                              const tipt_step_params* sp, const tipt_vsource* vp,
                              const double* sched, int64_t sched_len, const uint64_t* counter,
                              int64_t offset, void* stream);

/* tipt_rk2_step_table_sched on an expanding background (the reference's
 * HUBBLE_EXPANSION loop, R:3621-3636): sched holds sched_len rows
 * (T, ns, eta_eff, inv_a2), and a step reads its eta_eff = eta + 3H/mu and
 * inv_a2 = 1/a^2 from its row in place of sp->eta_eff and sp->inv_a2. */
int tipt_rk2_step_table_sched4(int storage, const void* phi, const void* pi, void* phi_out,
                               void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                               const tipt_step_params* sp, const tipt_vsource* vp,
                               const double* sched, int64_t sched_len, const uint64_t* counter,
                               int64_t offset, void* stream);

/* *counter += k on the stream (one-thread kernel; graph-capturable). */
int tipt_counter_add(uint64_t* counter, int64_t k, void* stream);

/* rk2_fused_table (R:1708-1872): two dt/2 midpoint halves, the first with
 * vp_T, the second with vp_Tm; array noise adds 0.5*noise in each half
 * (R:1806, R:1872).  With noise == NULL the halves use the inline hash of
 * rk2_fused_single_pass: 0.5*ns*z at multiplier 73856093, then 19349669
 * (R:2511-2522, R:2636-2647).  mid_phi / mid_pi hold the state between the
 * halves (the reference's phi_tmp / pi_tmp). */
int tipt_rk2_fused_table(int storage, const void* phi, const void* pi, void* phi_out,
                         void* pi_out, void* mid_phi, void* mid_pi, int64_t nx, int64_t ny,
                         int64_t nz, const tipt_step_params* sp, const tipt_vsource* vp_T,
                         const tipt_vsource* vp_Tm, const void* noise, void* stream);

/* Allocation-free form of tipt_rk2_fused_table, for callers that cannot
 * allocate device memory (code running inside another library's CUDA-graph
 * capture, hosts without a device allocator, real-time loops).  No counterpart
 * in the reference.  The intermediate state lives in an 8 MiB device array
 * inside the library (held by every GPU that loads it until exit); lattices
 * whose intermediate phi and pi exceed it (about 512K sites for F64 / F32C,
 * 1M for F32) are rejected with TIPT_ERR_UNSUPPORTED.  All calls share the
 * array: calls that overlap on the GPU race.  The first call on each device
 * looks up the array's device address and should precede any stream capture.
 * Allocates nothing. */
int tipt_rk2_fused_table_noalloc(int storage, const void* phi, const void* pi, void* phi_out,
                                 void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                                 const tipt_step_params* sp, const tipt_vsource* vp_T,
                                 const tipt_vsource* vp_Tm, const void* noise, void* stream);

/* --------------------------------------------------------- complex field */

/* Complex rk2_step_table (C:2067-2215): the real step for Phi = phi1 + i phi2
 * with V'(rho) from vp (rho = |Phi|), projected onto the components
 * (C:2137-2139), plus the terms in ct.  Array noise: noise1 / noise2 as the
 * reference passes them; NULL: one hash pair per site, z1 = r cos -> pi1,
 * z2 = r sin -> pi2 (C:2958-2974). */
int tipt_complex_rk2_step_table(int storage, const void* phi1, const void* phi2,
                                const void* pi1, const void* pi2, void* phi1_out,
                                void* phi2_out, void* pi1_out, void* pi2_out, int64_t nx,
                                int64_t ny, int64_t nz, const tipt_step_params* sp,
                                const tipt_vsource* vp, const tipt_complex_terms* ct,
                                const void* noise1, const void* noise2, void* stream);

/* tipt_complex_rk2_step_table that also reports the range of the new |Phi|
 * (the complex loop's per-step rho check, C:4263-4288) without a pass of its
 * own: range / range_next as in tipt_rk2_step_table_range, folded from
 * rho = sqrt(phi1^2 + phi2^2) of the values written (FP32; compensated FP32:
 * hi + lo; FP64: computed in FP64, rounded to FP32). */
int tipt_complex_rk2_step_table_range(int storage, const void* phi1, const void* phi2,
                                      const void* pi1, const void* pi2, void* phi1_out,
                                      void* phi2_out, void* pi1_out, void* pi2_out, int64_t nx,
                                      int64_t ny, int64_t nz, const tipt_step_params* sp,
                                      const tipt_vsource* vp, const tipt_complex_terms* ct,
                                      const void* noise1, const void* noise2, uint32_t* range,
                                      uint32_t* range_next, void* stream);

/* Complex rk2_fused_table (C:1789-2064): two dt/2 midpoint halves, the first
 * with vp_T, the second with vp_Tm; array noise adds 0.5*noise_a in each half.
 * With noise1 == noise2 == NULL the halves use the inline hash pairs of the
 * complex rk2_fused_single_pass (C:2765-3132): 0.5*ns*(z1, z2) at multiplier
 * 73856093, then 19349669.  vp_T / vp_Tm may be TIPT_VP_THERMAL (the inline
 * V'(rho) of C:2605-2680).  mid1..mid4 hold the state between the halves (the
 * reference's phi1_tmp .. pi2_tmp); the outputs may be the inputs. */
int tipt_complex_rk2_fused_table(int storage, const void* phi1, const void* phi2,
                                 const void* pi1, const void* pi2, void* phi1_out,
                                 void* phi2_out, void* pi1_out, void* pi2_out, void* mid1,
                                 void* mid2, void* mid3, void* mid4, int64_t nx, int64_t ny,
                                 int64_t nz, const tipt_step_params* sp, const tipt_vsource* vp_T,
                                 const tipt_vsource* vp_Tm, const tipt_complex_terms* ct,
                                 const void* noise1, const void* noise2, void* stream);

/* compute_winding_number (C:2683-2744; tools/winding.py:15-64) on the FP64
 * value of the stored fields (the reference casts to FP64, C:4627-4629).
 * Outputs (each may be NULL):
 *   w_site[N] float   -- sum over the XY, XZ, YZ plaquettes anchored at the
 *                         site, each plaquette's integer winding (the
 *                         reference's float value rounded),
 *   w3[3][N] int8     -- per-orientation integer windings (XY, XZ, YZ),
 *   pierced[cap] uint32 -- compacted list of pierced plaquettes, entry =
 *                         site*3 + orientation, in no particular order,
 *   counts[5] int64   -- device: pierced XY, XZ, YZ; sites with |w| > 0.5
 *                         (the reference string count, C:4661); list length
 *                         written (<= cap).  Zeroed by the call. */
int tipt_compute_winding_number(int storage, const void* phi1, const void* phi2, int64_t nx,
                                int64_t ny, int64_t nz, float* w_site, int8_t* w3,
                                uint32_t* pierced, int64_t pierced_cap, int64_t* counts,
                                void* stream);

/* -------------------------------------------------------------- ensemble */

/* One replica of a batched ensemble (no reference counterpart: the reference
 * runs one lattice per invocation).  Replicas are slices of one packed state
 * buffer (planar hi/lo for TIPT_F32C over all n_total sites).  A 2-D lattice
 * is given as (1, nx, ny). */
typedef struct {
    int32_t n0, n1, n2;  /* extents; n2 contiguous */
    uint32_t m1, m2;     /* ceil(2^32 / n1), ceil(2^32 / n2); 0 for an extent of 1 */
    int32_t pad_;
    int64_t offset;      /* first site of the replica in the packed buffers */
    double c1, c2, c3;   /* V'(phi) = c1 phi + c2 phi^2 + c3 phi^3 */
    double noise_scale;  /* ns: kick ns*z per step (R:3714-3718) */
    uint64_t seed;       /* hash noise seed of the replica */
} tipt_replica;

/* A work-list entry: sites [begin, begin + count) of one replica. */
typedef struct {
    int32_t replica;
    int32_t count;
    int64_t begin;
} tipt_chunk;

/* One midpoint RK2 step (the rk2_step_table arithmetic, R:1875-1966, with a
 * polynomial V' and inline hash noise) of every active replica, as one
 * persistent launch over the chunk work-list; replicas with active[r] == 0 are
 * skipped.  sp supplies dt, dx, eta_eff, mu, inv_a2; the hash step is
 * sp->noise_step, plus *counter + offset when counter (a device uint64) is
 * given (graph-captured loops). */
int tipt_ensemble_step(int storage, const void* phi, const void* pi, void* phi_out, void* pi_out,
                       int64_t n_total, const tipt_replica* replicas, const tipt_chunk* chunks,
                       int32_t n_chunks, const int32_t* active, const tipt_step_params* sp,
                       const uint64_t* counter, int64_t offset, void* stream);

/* The same step for the replicas rids[0..n_rids) of one 3-D shape class
 * (n0 x n1 x n2, n2 % 4 == 0, n0 >= 2), compensated-FP32 storage, on the
 * marching stage (shared-memory tiles fed by bulk copies); bitwise equal to
 * tipt_ensemble_step for those replicas.  The packed buffers (and n_total * 4
 * bytes) must be 16-byte aligned; the replicas' offsets multiples of 4 sites. */
int tipt_ensemble_march_supported(int32_t n0, int32_t n1, int32_t n2);  /* 1 or 0 */
int tipt_ensemble_step_march(const void* phi, const void* pi, void* phi_out, void* pi_out,
                             int64_t n_total, const tipt_replica* replicas, const int32_t* rids,
                             int32_t n_rids, const int32_t* n_rids_dev, int32_t n0, int32_t n1,
                             int32_t n2, const int32_t* active, const tipt_step_params* sp,
                             const uint64_t* counter, int64_t offset, void* stream);
/* n_rids_dev (optional, a device int32 <= n_rids): the number of rids to step,
 * read by the launch -- with tipt_ensemble_compact the class's work items then
 * cover its active replicas only, spread over the SMs.  Ordered compaction:
 * rids_out[0..*n_out) = the rids[q] whose active flag is set. */
int tipt_ensemble_compact(const int32_t* rids, int32_t n, const int32_t* active,
                          int32_t* rids_out, int32_t* n_out, void* stream);

/* Per replica (one block each, fixed order): frac_out[r] = fraction of sites
 * with phi > thr.  An active replica whose fraction exceeds stop_frac for the
 * first time gets first_step[r] = step (+ *counter + offset; first_step starts
 * at -1); once its fraction exceeds retire_frac (>= stop_frac) it is retired:
 * active[r] = 0 and *n_active is decremented. */
int tipt_ensemble_observe(int storage, const void* phi, int64_t n_total,
                          const tipt_replica* replicas, int32_t n_replicas, int32_t* active,
                          int32_t* n_active, double thr, double stop_frac, double retire_frac,
                          uint64_t step,
                          const uint64_t* counter, int64_t offset, int64_t* first_step,
                          double* frac_out, void* stream);

/* ----------------------------------------------------------- observables */

/* compute_energy_densities (R:2270-2319) plus the host loop's per-step
 * reductions (phi.min/max R:3655-3660, NaN guard R:3882-3944) and the
 * converted fraction: out[10] (device, double) = E_kin, E_grad, E_pot,
 * <phi>, <phi^2>, <pi^2>, fraction(phi > thr), min phi, max phi,
 * non-finite count.  FP64 accumulation in a fixed order (deterministic for
 * given sizes).  workspace: caller-owned device memory of
 * tipt_observables_workspace_size(nx, ny, nz) bytes.  pi may be NULL. */
int64_t tipt_observables_workspace_size(int64_t nx, int64_t ny, int64_t nz);
int tipt_observables(int storage, const void* phi, const void* pi, int64_t nx, int64_t ny,
                     int64_t nz, double dx, double inv_a2, double lam, double mphi, double mu,
                     double thr, double* out, void* workspace, int64_t workspace_bytes,
                     void* stream);

/* tipt_observables over the computed planes 1..nx_local of a slab laid out as
 * for tipt_rk2_step_table_slab (the forward difference of the last plane reads
 * the upper ghost plane): means are divided by n_global_sites, so the sums over
 * ranks of out[0..6] and out[9] and the min / max over ranks of out[7] / out[8]
 * give the lattice's observables.  workspace: tipt_observables_workspace_size(
 * nx_local + 2, ny, nz) bytes. */
int tipt_observables_slab(int storage, const void* phi, const void* pi, int64_t nx_local,
                          int64_t ny, int64_t nz, int64_t n_global_sites, double dx,
                          double inv_a2, double lam, double mphi, double mu, double thr,
                          double* out, void* workspace, int64_t workspace_bytes, void* stream);

/* ------------------------------------------------------------ other integrators
 * The reference's alternative integrators with counter-based hash noise (key
 * of (site, noise_step) at the pass-2 multiplier, seed noise_seed).  The
 * reference updates in place inside a parallel loop; here each sub-step reads
 * the previous sub-step's state only (outputs must not overlap inputs).
 * Storages F64, F32 (the reference's float32 mode), F32C; V' a 1-D table or a
 * polynomial. */

/* R:2115 overdamped_euler_step_table: phi_out = phi + dt/eta_eff F(phi) +
 * noise_scale z, F = inv_a2 lap(phi) - V'(phi)/mu^2. */
int tipt_overdamped_step_table(int storage, const void* phi, void* phi_out, int64_t nx,
                               int64_t ny, int64_t nz, const tipt_step_params* sp,
                               const tipt_vsource* vp, void* stream);

/* R:1974 baoab_step_table: B A O A B with gamma = sp->eta_eff, c1 = exp(-gamma dt),
 * c2 = sqrt(1 - c1^2) noise_scale; two launches (the second updates pi_out in
 * place). */
int tipt_baoab_step_table(int storage, const void* phi, const void* pi, void* phi_out,
                          void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                          const tipt_step_params* sp, const tipt_vsource* vp, void* stream);

/* C:2422 / C:2223: the same for the complex field (V'(rho) projected, Z_N and
 * eps Re Phi^4 from ct; the two components take the cosine and sine branches
 * of one Box-Muller pair). */
int tipt_complex_overdamped_step_table(int storage, const void* phi1, const void* phi2,
                                       void* phi1_out, void* phi2_out, int64_t nx, int64_t ny,
                                       int64_t nz, const tipt_step_params* sp,
                                       const tipt_vsource* vp, const tipt_complex_terms* ct,
                                       void* stream);
int tipt_complex_baoab_step_table(int storage, const void* phi1, const void* phi2,
                                  const void* pi1, const void* pi2, void* phi1_out,
                                  void* phi2_out, void* pi1_out, void* pi2_out, int64_t nx,
                                  int64_t ny, int64_t nz, const tipt_step_params* sp,
                                  const tipt_vsource* vp, const tipt_complex_terms* ct,
                                  void* stream);

/* ------------------------------------------------------------ thermal V'
 * The physics-default thermal potential (R:432-496, R:755-849, R:1415-1485):
 * V'(phi, T) = lam phi^3 - mphi^2 phi + T^4/(2 pi^2) (cb dJ_B(u_b) du_b/dphi +
 * cf dJ_F(u_f) du_f/dphi), u_b = sqrt(mB^2 + gb^2 phi^2 / 2 + (gb^2/4 + 2 gg^2/3) T^2) / T,
 * u_f = sqrt(gf^2 phi^2 / 2 + gfg^2 T^2 / 6) / T, dJ from cubic splines on a
 * uniform u grid. */
typedef struct tipt_thermal {
    double lam, mphi, boson_mass_sq;
    double boson_coupling, boson_gauge_coupling, fermion_coupling, fermion_gauge_coupling;
    double coeff_b, coeff_f;  /* the reference's _POT_COEFFS */
    double x_min, h;          /* spline grid: u_i = x_min + i h, i = 0..nseg */
    int32_t nseg;
    int32_t form;             /* steppers' per-site V' (TIPT_VP_THERMAL): 0 = the inline form
                                 _vprime_inline (R:2201-2266: x clamped to
                                 x_min + h nseg - 1e-12, segment (x - x_min) * (1/h)),
                                 1 = the Vprime_field form (R:1435-1485 with
                                 cubic_eval_uniform R:1415-1426: clamped only above
                                 x_min + h nseg, segment (x - x_min) / h) */
    const double* spline;     /* device [8][nseg]: dx^3, dx^2, dx, 1 coefficients of dJ_B, then dJ_F */
} tipt_thermal;

/* dJ_B (fermion = 0) or dJ_F (1) at the n device points u (FP64 quadrature,
 * composite 16-point Gauss-Legendre; gl_nodes / gl_weights are HOST arrays of
 * the 16 nodes and weights on [-1, 1]); with x_cut > 0 the lattice
 * counterterm's soft-mode part (R:461-490) is subtracted. */
int tipt_thermal_dj(int fermion, const double* u, int32_t n, const double* gl_nodes,
                    const double* gl_weights, double x_cut, double* out, void* stream);

/* R:1435 Vprime_field: out[N] (FP64) = V'(phi, T) per site. */
int tipt_thermal_vprime_field(int storage, const void* phi, double T, const tipt_thermal* tp,
                              double* out, int64_t nx, int64_t ny, int64_t nz, void* stream);

/* R:805-849 build_vprime_table on a (phi, T) grid: out[nT][nphi] = V'(phi_i, T_j),
 * phi_i = linspace(phi_lo, phi_hi, nphi), T_j from the device array Ts. */
int tipt_thermal_vprime_table(double phi_lo, double phi_hi, int32_t nphi, const double* Ts,
                              int32_t nT, const tipt_thermal* tp, double* out, void* stream);

/* C:1452-1530 Vprime_field of the complex field: out1, out2 (FP64, N each) =
 * V'(rho_safe, T) phi_a / rho_safe with rho_safe = max(|phi|, 1e-30), the radial
 * V' of tipt_thermal_vprime_field, plus the Z_N term of ct (NULL: none). */
int tipt_thermal_vprime_field_complex(int storage, const void* phi1, const void* phi2, double T,
                                      const tipt_thermal* tp, const tipt_complex_terms* ct,
                                      double* out1, double* out2, int64_t nx, int64_t ny,
                                      int64_t nz, void* stream);

/* R:1364-1385 laplacian_periodic(out, a, dx): the periodic 7-point Laplacian
 * (a[ip] + a[im] + a[jp] + a[jm] + a[kp] + a[km] - 6 a) / dx^2 into out, which
 * has a's storage (F32: float32 neighbour sum, the rest in FP64, as the
 * reference on float32 arrays; F32C: FP64 from hi + lo, stored as a {hi, lo}
 * pair).  out must not overlap a. */
int tipt_laplacian_periodic(int storage, const void* a, void* out, int64_t nx, int64_t ny,
                            int64_t nz, double dx, void* stream);

/* R:1415-1426 cubic_eval_uniform(x, x_min, h, nseg, c0, c1, c2, c3) at the n
 * device points x: segment trunc((x - x_min) / h) clamped to [0, nseg - 1],
 * Horner in dx = x - (x_min + i h) with the device coefficient arrays c0 (dx^3)
 * .. c3 (1), FP64, into out[n]. */
int tipt_cubic_eval_uniform(const double* x, int64_t n, double x_min, double h, int32_t nseg,
                            const double* c0, const double* c1, const double* c2,
                            const double* c3, double* out, void* stream);

/* ------------------------------------------------------------ labelling
 * Connected components of |field| > threshold (face neighbours, open or
 * periodic lattice), numbered 1..n in raster order of each component's first
 * site: the label array of scipy.ndimage.label, which the reference's
 * post-processing uses for bubbles and string voxels
 * (postprocess/revisualize_snapshots.py:171-214, :360-392). */
int64_t tipt_label_workspace_size(int64_t nx, int64_t ny, int64_t nz);

/* labels[N] (int32, 0 = background) and *n_labels (device int32). */
int tipt_label_components(int storage, const void* field, double threshold, int64_t nx,
                          int64_t ny, int64_t nz, int periodic, int32_t* labels,
                          int32_t* n_labels, void* workspace, int64_t workspace_bytes,
                          void* stream);

/* Per-label sums over the sites of each label l in 1..n_labels (arrays of
 * n_labels + 1 entries, entry 0 unused): site count, sum of (i, j, k), sum of
 * i^2 + j^2 + k^2, sum of the field value and the largest |value| (field may
 * be NULL: value 0). */
int tipt_label_stats(int storage, const void* field, const int32_t* labels, int64_t nx,
                     int64_t ny, int64_t nz, int32_t n_labels, int64_t* count, int64_t* sum_xyz,
                     int64_t* sum_sq, double* sum_val, double* max_abs, void* stream);

/* ------------------------------------------------------------ surrogate network
 * No reference counterpart (the reference estimates nucleation only by running
 * lattices).  A 6 -> 128 -> 128 -> 128 -> 17 SiLU network maps normalised
 * (T/T0, E, D, lam, log volume, dimension) to the log nucleation rate (in
 * exposure units) and the logits of the converted fraction at 16 fixed times.
 * Parameters: one FP32 vector of tipt_mlp_param_count() values, per layer
 * W[in][out] then b[out] with layer widths 16, 128, 128, 128, 32 (inputs 6..15
 * and outputs 17..31 are padding and stay zero).  Products use BF16 operands
 * with FP32 accumulation on the tensor cores; results are deterministic. */
int64_t tipt_mlp_param_count(void);

/* Kernel selection for the network: 0 automatic (tcgen05 tensor-core kernels
 * with tensor-memory accumulators), 1 the mma.sync kernels, 2 tcgen05.  The two
 * paths differ only in FP32 accumulation order. */
int tipt_mlp_set_policy(int policy);

/* Bytes of device workspace tipt_mlp_grad needs for `rows` rows. */
int64_t tipt_mlp_workspace_size(int64_t rows);

/* y[rows][17] = network(x[rows][6]) (FP32, row-major). */
int tipt_mlp_forward(const float* params, const float* x, int64_t rows, float* y, void* stream);

/* Gradient of (1/norm) sum_rows loss(row) with respect to params into grad (FP32,
 * parameter layout); per-row losses into loss_rows when not NULL.  tgt[rows][20]
 * per row: event (1 if the replica's first passage happened), exposure (volume x
 * time to first passage or to censoring, in the units of the rate output),
 * w_gamma, w_curve, then the 16 converted fractions in [0, 1].  loss(row) =
 * w_gamma (exp(l) exposure - event l) + w_curve/16 sum_k (softplus(o_k) - f_k o_k),
 * l = y[0] clamped to [-40, 40] inside the exponential, o_k = y[k]. */
int tipt_mlp_grad(const float* params, const float* x, const float* tgt, int64_t rows,
                  float norm, float* grad, float* loss_rows, void* workspace,
                  int64_t workspace_bytes, void* stream);

/* One Adam step over all parameters (bias-corrected with step t = *counter +
 * offset + 1, or offset + 1 without a counter; decoupled weight decay).  The
 * learning rate is lr, times lr_schedule[min(t, schedule_len) - 1] when a
 * device schedule is given (graph-captured training loops). */
int tipt_mlp_adam(float* params, const float* grad, float* m, float* v, const uint64_t* counter,
                  int64_t offset, float lr, const float* lr_schedule, int64_t schedule_len,
                  float beta1, float beta2, float eps, float weight_decay, void* stream);

/* ------------------------------------------------------------ control */

/* Real-field stage kernel selection: 0 automatic (the TMA marching kernel where
 * the shape allows: contiguous extent a multiple of 4 in [8, 1024]), 1 the
 * generic one-site-per-thread kernel, 2 the marching kernel or an error.  Both
 * kernels produce bitwise identical results.  No reference counterpart
 * (the reference's only knob is the CPU tile size, R:1969-1970). */
int tipt_set_kernel_policy(int policy);

/* Marching-kernel tile shape: rows per tile, planes per work item and ring
 * stages (each 0 = automatic).  Performance only; used by the autotuner. */
int tipt_set_march_tiles(int rows, int planes, int stages);

/* Compensated-FP32 marching kernels compiled for a fixed geometry, used when the
 * automatic geometry is theirs: the real stage (rows of 512 sites in 4-row
 * tiles, 256 sites in 8-row tiles), the complex stage (256-site segments in
 * 4-row tiles), the integrators (512 sites, 4 rows) and the ensemble classes
 * (64 sites, 32 rows; 96 sites, 16 rows).  enable != 0 (the default) or 0 for
 * the run-time-geometry kernels.  Performance only: both give the same bits. */
int tipt_set_march_fixed(int enable);

/* Row segment of the complex marching kernel (sites per segment, a divisor of
 * nz of at least 128; 0 = automatic).  Performance only; used by the autotuner. */
int tipt_set_march_kseg(int kseg);

/* Device status word set by bounded device-side waits that expired
 * (TIPT_ERR_TIMEOUT), 0 otherwise; clear != 0 resets it.  Synchronises the
 * device.  Counterpart of the reference's host NaN/divergence guard in spirit
 * (R:3882-3944): failures are reported, never trapped. */
int tipt_device_status(int* status, int clear);

/* Test of the bounded device waits (no reference counterpart; the reference's
 * only failure handling is the host NaN guard, R:3882-3944): arms the next
 * compensated-FP32 marching stage launch to withhold ring position `position`
 * in its block 0, so that block's consumers wait for a plane that never
 * arrives, give up after the bounded wait (2 s), set TIPT_ERR_TIMEOUT and
 * return; nothing is left in flight.  One launch only; position < 0 disarms. */
int tipt_test_withhold_plane(int position);

#ifdef __cplusplus
}
#endif

#endif /* TIPT_H */
