// extern "C" entry points of libtipt.so (declared in include/tipt.h):
// argument validation, status codes and the mapping from the reference's
// call signatures onto the kernel launch parameters.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "rk2_real.cuh"
#include "tipt_internal.h"

namespace tipt {

static thread_local char g_err[512] = "";

int fail(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return status;
}

int fail_cuda(cudaError_t e, const char* what) {
    snprintf(g_err, sizeof(g_err), "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
    return TIPT_ERR_CUDA;
}

int launch_hash_pairs(const uint64_t*, int64_t, double*, double*, double*, cudaStream_t);
int launch_noise_fill(int, void*, int64_t, double, uint64_t, uint64_t, uint64_t, int,
                      cudaStream_t);

int check_dims(int64_t nx, int64_t ny, int64_t nz) {
    if (nx < 1 || ny < 1 || nz < 1)
        return fail(TIPT_ERR_ARG, "lattice extents must be >= 1, got (%lld, %lld, %lld)",
                    (long long)nx, (long long)ny, (long long)nz);
    if (nx > (1 << 30) || ny > (1 << 30) || nz > (1 << 30) ||
        (double)nx * (double)ny * (double)nz > 9.0e15)
        return fail(TIPT_ERR_ARG, "lattice too large");
    return TIPT_OK;
}

int check_storage(int s) {
    if (s != TIPT_F64 && s != TIPT_F32 && s != TIPT_F32C)
        return fail(TIPT_ERR_STORAGE, "unknown storage %d", s);
    return TIPT_OK;
}

// Bytes per site (F32C: a hi and a lo float) and required pointer alignment.
int elem_bytes(int s) { return s == TIPT_F32 ? 4 : 8; }
int elem_align(int s) { return s == TIPT_F64 ? 8 : 4; }

int check_ptr(const void* p, int align, const char* name) {
    if (!p) return fail(TIPT_ERR_ARG, "%s is NULL", name);
    if (reinterpret_cast<uintptr_t>(p) % align)
        return fail(TIPT_ERR_ALIGN, "%s is not %d-byte aligned", name, align);
    return TIPT_OK;
}

// Two byte ranges [a, a+n) and [b, b+n) overlap.
bool overlap(const void* a, const void* b, int64_t n) {
    const char* x = static_cast<const char*>(a);
    const char* y = static_cast<const char*>(b);
    return x < y + n && y < x + n;
}

int check_vsource(const tipt_vsource* vp, const char* name) {
    if (!vp) return fail(TIPT_ERR_ARG, "%s is NULL", name);
    if (vp->kind == TIPT_VP_POLY) return TIPT_OK;
    if (vp->kind == TIPT_VP_THERMAL) {
        const tipt_thermal* t = vp->thermal;
        if (!t) return fail(TIPT_ERR_ARG, "%s: thermal parameters are NULL", name);
        if (t->nseg < 1 || !(t->h > 0.0)) return fail(TIPT_ERR_ARG, "%s: bad spline grid", name);
        if (!t->spline || reinterpret_cast<uintptr_t>(t->spline) % 8)
            return fail(TIPT_ERR_ALIGN, "%s: spline is NULL or misaligned", name);
        if (!(vp->T > 0.0)) return fail(TIPT_ERR_ARG, "%s: T must be > 0", name);
        if (t->form != 0 && t->form != 1)
            return fail(TIPT_ERR_ARG, "%s: thermal form must be 0 (inline) or 1 (field)", name);
        return TIPT_OK;
    }
    if (vp->kind != TIPT_VP_TABLE && vp->kind != TIPT_VP_TABLE2D)
        return fail(TIPT_ERR_ARG, "%s: unknown V' source kind %d", name, vp->kind);
    if (!vp->table) return fail(TIPT_ERR_ARG, "%s: table is NULL", name);
    if (vp->npts < 2) return fail(TIPT_ERR_ARG, "%s: npts must be >= 2", name);
    if (vp->kind == TIPT_VP_TABLE2D && vp->nT < 2)
        return fail(TIPT_ERR_ARG, "%s: nT must be >= 2", name);
    return TIPT_OK;
}

static void fill_vsource(RealStageParams& p, const tipt_vsource* vp) {
    p.vkind = vp->kind;
    p.npts = vp->npts;
    p.table = vp->table;
    p.tmin = vp->tmin;
    p.dinv = vp->dinv;
    p.nT = vp->nT;
    p.T_min = vp->T_min;
    p.T_dinv = vp->T_dinv;
    p.T = vp->T;
    p.c1 = vp->c1;
    p.c2 = vp->c2;
    p.c3 = vp->c3;
    p.table_in_smem = 0;
    if (vp->kind == TIPT_VP_THERMAL) p.th = thermal_site(*vp->thermal, vp->T);
}

static RealStageParams stage_params(const void* phi, const void* pi, void* phi_out,
                                    void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                                    const tipt_step_params* sp, const tipt_vsource* vp) {
    RealStageParams p;
    memset(&p, 0, sizeof(p));
    p.phi = phi;
    p.pi = pi;
    p.phi_out = phi_out;
    p.pi_out = pi_out;
    p.n0 = (int)nx;
    p.n1 = (int)ny;
    p.n2 = (int)nz;
    p.inv_dx2 = 1.0 / (sp->dx * sp->dx);   // R:1898
    p.eta = sp->eta_eff;
    p.inv_mu2 = 1.0 / (sp->mu * sp->mu);   // R:1899
    p.inv_a2 = sp->inv_a2;
    p.step = sp->noise_step;
    p.seed = sp->noise_seed;
    fill_vsource(p, vp);
    return p;
}

int check_state(int storage, const void* phi, const void* pi, void* phi_out,
                       void* pi_out, int64_t nx, int64_t ny, int64_t nz) {
    int rc;
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz))) return rc;
    return check_state_sites(storage, phi, pi, phi_out, pi_out, nx * ny * nz);
}

int check_state_sites(int storage, const void* phi, const void* pi, void* phi_out,
                      void* pi_out, int64_t sites) {
    int rc;
    if ((rc = check_storage(storage))) return rc;
    if (sites < 1 || (double)sites > 9.0e15)
        return fail(TIPT_ERR_ARG, "site count %lld out of range", (long long)sites);
    const int eb = elem_bytes(storage), ea = elem_align(storage);
    if ((rc = check_ptr(phi, ea, "phi")) || (rc = check_ptr(pi, ea, "pi")) ||
        (rc = check_ptr(phi_out, ea, "phi_out")) || (rc = check_ptr(pi_out, ea, "pi_out")))
        return rc;
    const int64_t bytes = sites * eb;
    const void* ins[2] = {phi, pi};
    const void* outs[2] = {phi_out, pi_out};
    for (auto o : outs)
        for (auto i : ins)
            if (overlap(o, i, bytes))
                return fail(TIPT_ERR_ARG, "output state overlaps the input state (the fused "
                            "stage reads neighbours: ping-pong the buffers)");
    if (overlap(phi_out, pi_out, bytes)) return fail(TIPT_ERR_ARG, "phi_out overlaps pi_out");
    return TIPT_OK;
}

}  // namespace tipt

using namespace tipt;

extern "C" {

const char* tipt_version(void) { return "tipt 0.1 (sm_100a)"; }

const char* tipt_status_string(int s) {
    switch (s) {
        case TIPT_OK: return "ok";
        case TIPT_ERR_ARG: return "invalid argument";
        case TIPT_ERR_STORAGE: return "unsupported storage";
        case TIPT_ERR_ALIGN: return "misaligned pointer";
        case TIPT_ERR_CUDA: return "CUDA error";
        case TIPT_ERR_UNSUPPORTED: return "unsupported mode or size";
        case TIPT_ERR_TIMEOUT: return "device-side wait timed out";
    }
    return "unknown status";
}

const char* tipt_last_error(void) { return g_err; }

int tipt_hash_rng_pair(const uint64_t* keys, int64_t n, double* u1, double* u2, double* z,
                       void* stream) {
    if (n < 0) return fail(TIPT_ERR_ARG, "n < 0");
    if (n > 0 && !keys) return fail(TIPT_ERR_ARG, "keys is NULL");
    return launch_hash_pairs(keys, n, u1, u2, z, (cudaStream_t)stream);
}

int tipt_generate_noise_field(int out_storage, void* out, int64_t nx, int64_t ny, int64_t nz,
                              double scale, uint64_t step, uint64_t mul, uint64_t seed,
                              int component, void* stream) {
    int rc;
    if (out_storage != TIPT_F64 && out_storage != TIPT_F32)
        return fail(TIPT_ERR_STORAGE, "noise field storage must be F64 or F32");
    if ((rc = check_dims(nx, ny, nz)) || (rc = check_ptr(out, elem_bytes(out_storage), "out")))
        return rc;
    if (component != 0 && component != 1) return fail(TIPT_ERR_ARG, "component must be 0 or 1");
    return launch_noise_fill(out_storage, out, nx * ny * nz, scale, step, mul, seed, component,
                             (cudaStream_t)stream);
}

int tipt_rk2_step_table(int storage, const void* phi, const void* pi, void* phi_out,
                        void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                        const tipt_step_params* sp, const tipt_vsource* vp, const void* noise,
                        void* stream) {
    int rc;
    if ((rc = check_state(storage, phi, pi, phi_out, pi_out, nx, ny, nz))) return rc;
    if (!sp) return fail(TIPT_ERR_ARG, "step params are NULL");
    if ((rc = check_vsource(vp, "vp"))) return rc;
    if (noise && (rc = check_ptr(noise, storage == TIPT_F32 ? 4 : 8, "noise"))) return rc;
    RealStageParams p = stage_params(phi, pi, phi_out, pi_out, nx, ny, nz, sp, vp);
    p.h1 = 0.5 * sp->dt;  // R:1900 half_dt
    p.h2 = sp->dt;
    p.noise = noise;
    p.nfac = 1.0;
    p.ns_eff = sp->noise_scale;
    p.mul = kPass2Mul;
    return launch_real_stage(storage, p, (cudaStream_t)stream);
}

int tipt_rk2_step_table_range(int storage, const void* phi, const void* pi, void* phi_out,
                              void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                              const tipt_step_params* sp, const tipt_vsource* vp,
                              const void* noise, uint32_t* range, uint32_t* range_next,
                              void* stream) {
    int rc;
    if ((rc = check_state(storage, phi, pi, phi_out, pi_out, nx, ny, nz))) return rc;
    if (!sp) return fail(TIPT_ERR_ARG, "step params are NULL");
    if ((rc = check_vsource(vp, "vp"))) return rc;
    if (noise && (rc = check_ptr(noise, storage == TIPT_F32 ? 4 : 8, "noise"))) return rc;
    if ((rc = check_ptr(range, 4, "range")) || (rc = check_ptr(range_next, 4, "range_next")))
        return rc;
    if (overlap(range, range_next, 12)) return fail(TIPT_ERR_ARG, "range and range_next overlap");
    RealStageParams p = stage_params(phi, pi, phi_out, pi_out, nx, ny, nz, sp, vp);
    p.h1 = 0.5 * sp->dt;
    p.h2 = sp->dt;
    p.noise = noise;
    p.nfac = 1.0;
    p.ns_eff = sp->noise_scale;
    p.mul = kPass2Mul;
    p.range = reinterpret_cast<unsigned int*>(range);
    p.range_next = reinterpret_cast<unsigned int*>(range_next);
    return launch_real_stage(storage, p, (cudaStream_t)stream);
}

int tipt_rk2_step_table_slab_planes(int storage, const void* phi, const void* pi, void* phi_out,
                                    void* pi_out, int64_t nx_local, int64_t ny, int64_t nz,
                                    int64_t i_lo, int64_t nx_global, int64_t plane_begin,
                                    int64_t plane_end, const tipt_step_params* sp,
                                    const tipt_vsource* vp, void* stream) {
    int rc;
    if (nx_local < 1 || nz < 2) return fail(TIPT_ERR_ARG, "slab needs nx_local >= 1 and nz >= 2");
    if (i_lo < 0 || i_lo + nx_local > nx_global)
        return fail(TIPT_ERR_ARG, "slab planes [%lld, %lld) outside the %lld-plane lattice",
                    (long long)i_lo, (long long)(i_lo + nx_local), (long long)nx_global);
    if (plane_begin < 1 || plane_end > nx_local + 1 || plane_begin >= plane_end)
        return fail(TIPT_ERR_ARG, "array planes [%lld, %lld) not inside [1, %lld)",
                    (long long)plane_begin, (long long)plane_end, (long long)(nx_local + 1));
    if ((rc = check_state(storage, phi, pi, phi_out, pi_out, nx_local + 2, ny, nz))) return rc;
    if (!sp) return fail(TIPT_ERR_ARG, "step params are NULL");
    if ((rc = check_vsource(vp, "vp"))) return rc;
    RealStageParams p = stage_params(phi, pi, phi_out, pi_out, nx_local + 2, ny, nz, sp, vp);
    p.h1 = 0.5 * sp->dt;
    p.h2 = sp->dt;
    p.noise = nullptr;
    p.nfac = 1.0;
    p.ns_eff = sp->noise_scale;
    p.mul = kPass2Mul;
    p.i_begin = (int)plane_begin;
    p.i_end = (int)plane_end;
    p.site_offset = (long long)(i_lo - 1) * ny * nz;  // array plane 1 = lattice plane i_lo
    return launch_real_stage(storage, p, (cudaStream_t)stream);
}

int tipt_rk2_step_table_slab(int storage, const void* phi, const void* pi, void* phi_out,
                             void* pi_out, int64_t nx_local, int64_t ny, int64_t nz, int64_t i_lo,
                             int64_t nx_global, const tipt_step_params* sp,
                             const tipt_vsource* vp, void* stream) {
    return tipt_rk2_step_table_slab_planes(storage, phi, pi, phi_out, pi_out, nx_local, ny, nz,
                                           i_lo, nx_global, 1, nx_local + 1, sp, vp, stream);
}

static int step_table_sched(int storage, const void* phi, const void* pi, void* phi_out,
                            void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                            const tipt_step_params* sp, const tipt_vsource* vp,
                            const double* sched, int cols, int64_t sched_len,
                            const uint64_t* counter, int64_t offset, void* stream) {
    int rc;
    if ((rc = check_state(storage, phi, pi, phi_out, pi_out, nx, ny, nz))) return rc;
    if (!sp) return fail(TIPT_ERR_ARG, "step params are NULL");
    if ((rc = check_vsource(vp, "vp"))) return rc;
    if (vp->kind == TIPT_VP_THERMAL)
        return fail(TIPT_ERR_UNSUPPORTED, "scheduled steps take a table or a polynomial V'");
    if ((rc = check_ptr(sched, 8, "sched")) || (rc = check_ptr(counter, 8, "counter"))) return rc;
    if (sched_len < 1 || offset < 0) return fail(TIPT_ERR_ARG, "bad schedule length or offset");
    RealStageParams p = stage_params(phi, pi, phi_out, pi_out, nx, ny, nz, sp, vp);
    p.h1 = 0.5 * sp->dt;
    p.h2 = sp->dt;
    p.noise = nullptr;
    p.nfac = 1.0;
    p.ns_eff = 0.0;
    p.mul = kPass2Mul;
    p.sched = sched;
    p.ctr = reinterpret_cast<const unsigned long long*>(counter);
    p.offset = offset;
    p.sched_len = sched_len;
    p.sched_cols = cols;
    p.ns_mult = 1.0;
    return launch_real_stage(storage, p, (cudaStream_t)stream);
}

int tipt_rk2_step_table_sched(int storage, const void* phi, const void* pi, void* phi_out,
                              void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                              const tipt_step_params* sp, const tipt_vsource* vp,
                              const double* sched, int64_t sched_len, const uint64_t* counter,
                              int64_t offset, void* stream) {
    return step_table_sched(storage, phi, pi, phi_out, pi_out, nx, ny, nz, sp, vp, sched, 2,
                            sched_len, counter, offset, stream);
}

int tipt_rk2_step_table_sched4(int storage, const void* phi, const void* pi, void* phi_out,
                               void* pi_out, int64_t nx, int64_t ny, int64_t nz,
                               const tipt_step_params* sp, const tipt_vsource* vp,
                               const double* sched, int64_t sched_len, const uint64_t* counter,
                               int64_t offset, void* stream) {
    return step_table_sched(storage, phi, pi, phi_out, pi_out, nx, ny, nz, sp, vp, sched, 4,
                            sched_len, counter, offset, stream);
}

__global__ void counter_add_kernel(unsigned long long* c, long long k) { *c += (unsigned long long)k; }

int tipt_counter_add(uint64_t* counter, int64_t k, void* stream) {
    int rc;
    if ((rc = check_ptr(counter, 8, "counter"))) return rc;
    counter_add_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<unsigned long long*>(counter), (long long)k);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "counter_add launch");
}

int tipt_rk2_fused_table(int storage, const void* phi, const void* pi, void* phi_out,
                         void* pi_out, void* mid_phi, void* mid_pi, int64_t nx, int64_t ny,
                         int64_t nz, const tipt_step_params* sp, const tipt_vsource* vp_T,
                         const tipt_vsource* vp_Tm, const void* noise, void* stream) {
    int rc;
    if ((rc = check_state(storage, phi, pi, mid_phi, mid_pi, nx, ny, nz)) ||
        (rc = check_state(storage, mid_phi, mid_pi, phi_out, pi_out, nx, ny, nz)))
        return rc;
    if (!sp) return fail(TIPT_ERR_ARG, "step params are NULL");
    if ((rc = check_vsource(vp_T, "vp_T")) || (rc = check_vsource(vp_Tm, "vp_Tm"))) return rc;
    if (noise && (rc = check_ptr(noise, storage == TIPT_F32 ? 4 : 8, "noise"))) return rc;
    // first half at T (R:1742-1806), multiplier of pass 2
    RealStageParams a = stage_params(phi, pi, mid_phi, mid_pi, nx, ny, nz, sp, vp_T);
    a.h1 = a.h2 = 0.5 * sp->dt;
    a.noise = noise;
    a.nfac = 0.5;
    a.ns_eff = 0.5 * sp->noise_scale;
    a.mul = kPass2Mul;
    if ((rc = launch_real_stage(storage, a, (cudaStream_t)stream))) return rc;
    // second half at T_mid (R:1808-1872), multiplier of pass 4
    RealStageParams b = stage_params(mid_phi, mid_pi, phi_out, pi_out, nx, ny, nz, sp, vp_Tm);
    b.h1 = b.h2 = 0.5 * sp->dt;
    b.noise = noise;
    b.nfac = 0.5;
    b.ns_eff = 0.5 * sp->noise_scale;
    b.mul = kPass4Mul;
    return launch_real_stage(storage, b, (cudaStream_t)stream);
}

}  // extern "C"
