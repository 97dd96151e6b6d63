// Marching (2.5-D blocked) real-field midpoint stage for 8-byte storages
// (F32C float2 pairs and F64), the bandwidth kernel of the stepper.
//
// Work item = (j-block of TJ rows, i-chunk of CI planes); a CTA owns full rows
// along the contiguous axis n2, so the k-direction wrap stays inside shared
// memory.  Per plane the CTA needs TJ+2 rows (one halo row each side, rows
// taken modulo n1 = periodic wrap in j) of phi and pi.
//
// Warp roles.  The last warp is the producer: one lane loads each plane into
// an S-stage ring.  Real fields: the tile's rows of a plane are consecutive
// rows of the field in global memory (and, with the pitch equal to the row
// length, in shared memory), so each field component is one 1-D bulk copy
// (cp.async.bulk) per run of rows -- at most three runs where the tile wraps
// in j -- four to twelve copies per plane instead of one per row and box; the
// producer's issue rate bounds the stage when copies are small.  The complex
// kernel copies row segments with TMA tensor boxes (cp.async.bulk.tensor.3d,
// every coordinate reduced modulo its extent).  Stage s has a `full` mbarrier
// (producer's expect-tx arrival + the copy bytes) and an `empty` mbarrier (one
// arrival per consumer warp).  Consumer warps compute plane i from the ring
// (planes i-1, i, i+1: i, j and k neighbours) and release plane i-1 as soon
// as they have read it; there is no CTA-wide barrier in the loop, so warps
// drift freely within the ring's slack.  A consumer thread of the FP64 kernel
// owns the site pairs {2t, 2t+1} and {n2/2 + 2t, n2/2 + 2t + 1} of its row, of
// the F32C kernel four consecutive sites, so the 16-byte shared loads and
// global stores of a warp are contiguous.
//
// Every mbarrier wait is bounded by the global timer (2 s); on expiry the
// thread records TIPT_ERR_TIMEOUT in a device status word and returns; the
// producer drains the copies it issued (bounded) before it exits.
#include <cuda.h>

#include "integrators.cuh"
#include "rk2_march.cuh"
#include "tipt_internal.h"

namespace tipt {

__device__ int g_device_status = 0;  // 0 ok; TIPT_ERR_TIMEOUT after a wait expired

constexpr uint64_t kWaitNs = 2000000000ull;

// ---------------------------------------------------------------- PTX -----
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: true when the phase completed, false after kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_test(bar, parity))
        if (global_ns() - t0 > kWaitNs) return false;
    return true;
}
__device__ __forceinline__ void tma_row(void* dst, const CUtensorMap* tm, int k, int j, int i,
                                        uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(k), "r"(j), "r"(i), "r"(smem_addr(bar))
        : "memory");
}

// 1-D bulk copy global -> shared (addresses 16-byte aligned, bytes a multiple
// of 16), completing on a transaction-count mbarrier.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Copies the tile rows j0-1 .. j0-1+rows-1 (taken modulo n1) of plane `plane`
// of a field into a [rows][pitch] block: runs of consecutive rows are one
// contiguous range in global memory, and in shared memory too when the pitch
// is the row length, so a run is one bulk copy (at most three runs: the wrap
// at j = 0 and at j = n1); otherwise one copy per row.
template <typename E>
__device__ __forceinline__ void copy_tile_rows(E* dst, const E* field, int64_t plane, int j0,
                                               int rows, int n1, int n2, int pitch, uint64_t* bar) {
    int rr = 0;
    while (rr < rows) {
        int jr = j0 - 1 + rr;
        jr = jr < 0 ? jr + n1 : (jr >= n1 ? jr - n1 : jr);
        int len = pitch == n2 ? min(rows - rr, n1 - jr) : 1;
        bulk_copy(dst + (size_t)rr * pitch, field + (plane * n1 + jr) * n2,
                  (uint32_t)(len * n2 * (int)sizeof(E)), bar);
        rr += len;
    }
}

// -------------------------------------------------------------- params -----
struct MarchGeom {
    int TJ;        // rows per tile
    int CI;        // planes per i-chunk
    int BK;        // TMA box width (elements), divides n2
    int pitch;     // shared-memory row pitch (elements); pitch*8 is a multiple of 128
    int S;         // ring stages
    int nJB, nIC;  // j-blocks, i-chunks
    int items;
    int tab_bytes;    // staged V' row (bytes, 128-aligned)
    int stage_bytes;  // one ring stage: phi and pi tiles
    // compensated-FP32 single-lattice stage only: 1 = each CTA takes an equal
    // share of the nJB x planes (j-block, plane) units, j-block major, as one or
    // more runs of planes (items is then the number of units); 0 = items of CI
    // planes.  Every geometry starts with 0; only launch_f32c_stage sets it.
    int bal = 0;
    // complex kernel: rows split into nKS segments of KS sites (with nKS > 1 the
    // k-1 / k+1 neighbours of a segment's end sites are copied by the edge
    // threads); halo_off = bytes of the eight plane blocks of a stage
    int KS, nKS, halo_off;
};

template <int S>
struct MarchElem;
template <>
struct MarchElem<TIPT_F64> {
    using E = double;
    using TT = double;
};
// The reference's float32 mode: float32 planes, the FP64 V' table (R:1914-1933).
template <>
struct MarchElem<TIPT_F32> {
    using E = float;
    using TT = double;
};

// Pair loads/stores of two consecutive elements (16 bytes for 8-byte elements,
// 8 bytes for 4-byte ones).
template <typename E>
__device__ __forceinline__ void ld_pair_s(const E* p, E& a, E& b) {
    if constexpr (sizeof(E) == 8) {
        const float4 v = *reinterpret_cast<const float4*>(p);
        a = *reinterpret_cast<const E*>(&v.x);
        b = *reinterpret_cast<const E*>(&v.z);
    } else {
        const float2 v = *reinterpret_cast<const float2*>(p);
        a = v.x;
        b = v.y;
    }
}
template <typename E>
__device__ __forceinline__ void st_pair_g(E* p, const E& a, const E& b) {
    if constexpr (sizeof(E) == 8) {
        float4 v;
        *reinterpret_cast<E*>(&v.x) = a;
        *reinterpret_cast<E*>(&v.z) = b;
        *reinterpret_cast<float4*>(p) = v;
    } else {
        *reinterpret_cast<float2*>(p) = make_float2(a, b);
    }
}
template <typename E>
__device__ __forceinline__ void ld_pair_g(const E* p, E& a, E& b) {
    if constexpr (sizeof(E) == 8) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(p));
        a = *reinterpret_cast<const E*>(&v.x);
        b = *reinterpret_cast<const E*>(&v.z);
    } else {
        const float2 v = __ldg(reinterpret_cast<const float2*>(p));
        a = v.x;
        b = v.y;
    }
}

template <int S>
__device__ __forceinline__ void site_update(const RealStageParams& p, const void* s_tab,
                                            float, float, const typename MarchElem<S>::E ph[7],
                                            const typename MarchElem<S>::E pv[7], double noise,
                                            typename MarchElem<S>::E& a,
                                            typename MarchElem<S>::E& b) {
    if constexpr (S == TIPT_F64) update_f64(p, static_cast<const double*>(s_tab), ph, pv, noise, a, b);
    else update_f32(p, static_cast<const double*>(s_tab), ph, pv, noise, a, b);
}

// Launch bounds of the two block-size classes: up to 256 consumer threads
// (two CTAs per SM) or up to 512 (one CTA per SM), plus the producer warp.
// Ring position -> (stage, phase parity), advanced incrementally.
struct RingPos {
    uint32_t stage, phase;
    __device__ __forceinline__ void next(uint32_t ns) {
        if (++stage == ns) {
            stage = 0;
            phase ^= 1u;
        }
    }
};

// 17-18 warps per SM must fit the four 16K-register sub-partitions.
constexpr int kMarchRegs = 96;

template <int S, bool WIDE>
__global__ void __maxnreg__(kMarchRegs)
    rk2_stage_march(RealStageParams p_in, MarchGeom g) {
    RealStageParams p = p_in;
    resolve_schedule(p);
    using E = typename MarchElem<S>::E;
    using TT = typename MarchElem<S>::TT;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // carve from a 128-byte aligned base (TMA destinations need 128-byte
    // alignment; the allocation carries 128 bytes of slack for this)
    unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
    TT* s_tab = reinterpret_cast<TT*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + g.tab_bytes);
    uint64_t* empty = full + 8;
    unsigned char* ring = smem + g.tab_bytes + 128;

    const int n0 = p.n0, n1 = p.n1, n2 = p.n2;
    const int pitch = g.pitch;
    const int TJ = g.TJ;
    const uint32_t NS = (uint32_t)g.S;
    const int rows = TJ + 2;
    const int tpr = n2 >> 2;          // consumer threads per row
    const int nc = TJ * tpr;          // consumer threads (a multiple of 32)
    const int t = threadIdx.x;

    if (t == 0) {
        for (uint32_t s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], nc / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (p.table_in_smem) stage_table<TT>(p, s_tab);  // ends with __syncthreads
    else __syncthreads();

    const size_t half_stage = (size_t)(g.stage_bytes >> 1);
    auto fld = [&](uint32_t stage, int f) -> E* {
        return reinterpret_cast<E*>(ring + (size_t)stage * g.stage_bytes + (size_t)f * half_stage);
    };

    // ------------------------------------------------------------ producer
    // Each item loads planes i0-1 .. i0+ni (ni + 2 ring positions).
    if (t >= nc) {
        if (t != nc) return;
        const uint32_t plane_tx = (uint32_t)(2 * rows * n2 * (int)sizeof(E));
        const E* const src_phi = static_cast<const E*>(p.phi);
        const E* const src_pi = static_cast<const E*>(p.pi);
        RingPos w{0, 0};
        uint32_t issued = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < g.items && ok; item += gridDim.x) {
            const int ic = item / g.nJB;
            const int j0 = (item - ic * g.nJB) * TJ, i0 = p.i_begin + ic * g.CI;
            const int npl = min(g.CI, p.i_end - i0) + 2;
            for (int q = 0; q < npl; ++q) {
                // stage w.stage last held position issued - NS, released in phase w.phase ^ 1
                if (issued >= NS && !mbar_wait(&empty[w.stage], w.phase ^ 1u)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&full[w.stage], plane_tx);
                int iw = i0 - 1 + q;
                iw = iw < 0 ? iw + n0 : (iw >= n0 ? iw - n0 : iw);
                copy_tile_rows(fld(w.stage, 0), src_phi, iw, j0, rows, n1, n2, pitch, &full[w.stage]);
                copy_tile_rows(fld(w.stage, 1), src_pi, iw, j0, rows, n1, n2, pitch, &full[w.stage]);
                ++issued;
                w.next(NS);
            }
        }
        if (!ok) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
        // keep the CTA alive until the last copies issued have landed (bounded):
        // walk back over the last min(NS, issued) positions
        RingPos d = w;
        for (uint32_t k = 0; k < NS && k < issued; ++k) {
            d.stage = d.stage == 0 ? NS - 1 : d.stage - 1;
            if (d.stage == NS - 1) d.phase ^= 1u;
            (void)mbar_wait(&full[d.stage], d.phase);
        }
        return;
    }

    // ----------------------------------------------------------- consumers
    const int lane = t & 31;
    const int r = 1 + t / tpr;               // own tile row (1..TJ)
    const int c = 2 * (t - (r - 1) * tpr);   // first column of pair A
    const int half = n2 >> 1;
    const int kmA = c == 0 ? n2 - 1 : c - 1;                  // left of pair A
    const int kpA = c + 2;                                    // right of pair A
    const int kmB = half + c - 1;                             // left of pair B
    const int kpB = half + c + 2 == n2 ? 0 : half + c + 2;    // right of pair B
    const float tminf = (float)p.tmin, dinvf = (float)p.dinv;
    E* const phi_out = static_cast<E*>(p.phi_out);
    E* const pi_out = static_cast<E*>(p.pi_out);
    const int orow = r * pitch, urow = (r - 1) * pitch, drow = (r + 1) * pitch;

    RingPos pm{0, 0};  // ring position of plane i-1 for the current iteration
    for (int item = blockIdx.x; item < g.items; item += gridDim.x) {
        const int ic = item / g.nJB;
        const int j0 = (item - ic * g.nJB) * TJ, i0 = p.i_begin + ic * g.CI;
        const int ni = min(g.CI, p.i_end - i0);
        const int jw = j0 + r - 1;
        RingPos pc = pm, pp;
        pc.next(NS);
        pp = pc;
        pp.next(NS);
        if (!mbar_wait(&full[pm.stage], pm.phase) || !mbar_wait(&full[pc.stage], pc.phase)) {
            if (lane == 0) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
            return;
        }
        for (int q = 0; q < ni; ++q) {
            const int i = i0 + q;
            const int64_t rowoff = ((int64_t)i * n1 + jw) * n2;
            // the noise reads no tile: drawn before the wait for the next plane
            double nz[2][2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int col = (h ? half + c : c) + u;
                    uint64_t site;
                    if constexpr (WIDE) site = (uint64_t)(rowoff + p.site_offset + col);
                    else site = (uint32_t)(rowoff + p.site_offset) + (uint32_t)col;
                    nz[h][u] = site_noise<E>(p, site);
                }
            }
            if (!mbar_wait(&full[pp.stage], pp.phase)) {
                if (lane == 0) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
                return;
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {   // pair A (h = 0), pair B (h = 1)
                const int col = h ? half + c : c;
                const int kl_ = h ? kmB : kmA;
                const int kr_ = h ? kpB : kpA;
                E ce[2][2], ip[2][2], im[2][2], jp[2][2], jm[2][2], kl[2], kr[2];
#pragma unroll
                for (int f = 0; f < 2; ++f) {
                    const E* sc = fld(pc.stage, f);
                    ld_pair_s(sc + orow + col, ce[f][0], ce[f][1]);
                    ld_pair_s(sc + urow + col, jm[f][0], jm[f][1]);
                    ld_pair_s(sc + drow + col, jp[f][0], jp[f][1]);
                    kl[f] = sc[orow + kl_];
                    kr[f] = sc[orow + kr_];
                    ld_pair_s(fld(pm.stage, f) + orow + col, im[f][0], im[f][1]);
                    ld_pair_s(fld(pp.stage, f) + orow + col, ip[f][0], ip[f][1]);
                }
                if (h == 1) {  // this warp is done with plane i-1
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[pm.stage]);
                }
                E op[2], ov[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    // stencil order: centre, ip, im, jp, jm, kp, km (R:1913-1920)
                    const E ph[7] = {ce[0][u], ip[0][u], im[0][u], jp[0][u], jm[0][u],
                                     u ? kr[0] : ce[0][1], u ? ce[0][0] : kl[0]};
                    const E pv[7] = {ce[1][u], ip[1][u], im[1][u], jp[1][u], jm[1][u],
                                     u ? kr[1] : ce[1][1], u ? ce[1][0] : kl[1]};
                    site_update<S>(p, s_tab, tminf, dinvf, ph, pv, nz[h][u], op[u], ov[u]);
                }
                st_pair_g(phi_out + rowoff + col, op[0], op[1]);
                st_pair_g(pi_out + rowoff + col, ov[0], ov[1]);
            }
            pm = pc;
            pc = pp;
            pp.next(NS);
        }
        // planes i0+ni-1 and i0+ni were read for the last time
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&empty[pm.stage]);
            mbar_arrive(&empty[pc.stage]);
        }
        pm = pp;  // the next item starts at the following ring position
    }
}

// Batched-ensemble arguments of the compensated-FP32 marching stage (unused for
// a single lattice).
struct EnsMarch {
    const tipt_replica* reps;
    const int32_t* rids;          // the class's replica ids (its active ones, compacted)
    const int32_t* n_rids;        // device count of rids (nullptr: g.items covers them all)
    const int32_t* active;
    int64_t n_total;              // sites of the packed buffers
    int items_per_rep;            // work items of one replica
    uint64_t step;
    const unsigned long long* ctr;  // device step counter or nullptr
    long long offset;
};

// The runs of planes of one CTA under MarchGeom::bal: CTA b of G takes the units
// [U b / G, U (b + 1) / G) of the U = nJB x planes (j-block, plane) units, j-block
// major, split where a j-block ends.  Producer and consumers walk the same runs.
struct BalRun {
    int64_t u, u_end;
    int npl, i_begin;
    __device__ __forceinline__ BalRun(const MarchGeom& g, const RealStageParams& p, int b, int G) {
        npl = p.i_end - p.i_begin;
        i_begin = p.i_begin;
        const int64_t U = (int64_t)g.nJB * npl;
        u = g.bal ? U * b / G : 0;
        u_end = g.bal ? U * (b + 1) / G : 0;
    }
    __device__ __forceinline__ bool more() const { return u < u_end; }
    // the next run: j-block jb, first plane i0, ni planes
    __device__ __forceinline__ void next(int& jb, int& i0, int& ni) {
        jb = (int)(u / npl);
        const int off = (int)(u - (int64_t)jb * npl);
        ni = (int)min((int64_t)(npl - off), u_end - u);
        i0 = i_begin + off;
        u += ni;
    }
};

// Planar compensated-FP32 marching kernel.  Same ring, roles and work items as
// rk2_stage_march; a field is two FP32 planes (hi, then lo N sites later), so
// the TMA map spans 2*n0 planes and a ring stage holds [phi, pi][hi, lo]
// tiles.  A consumer thread owns four consecutive sites of its row (one
// 16-byte vector per plane and neighbour) and evaluates them as two site
// pairs in the lanes of the packed FP32x2 instructions; the stencil sums run
// in the order of the generic kernel, so results are bitwise identical.
//
// ENS: the replicas of one shape class of a batched ensemble (packed buffers:
// the hi planes of all n_total sites, then the lo planes), each with its own
// polynomial V', noise amplitude and seed; work items run over (replica,
// j-block, i-chunk) and both warp roles skip the items of retired replicas.
// The per-site arithmetic is the single-lattice kernel's, so a replica's
// result is bitwise that of the lattice stepped alone.
//
// KN2, KTJ > 0: the geometry fixed at compile time (rows of KN2 sites, pitch
// KN2, KTJ-row tiles), so every shared-memory offset but the ring stage's is an
// immediate and the row arithmetic is shifts; the launcher picks it when the
// run-time geometry is exactly that one.
// TAB: the V' source is the row staged in shared memory and the noise is the
// hash (no noise array), fixed at compile time: the per-site arithmetic then
// has no run-time branch on the source, which lets the compiler schedule the
// noise, lookups and update of a plane as one block (7-12 % faster than the
// run-time dispatch).  The same operations as the dispatching form.
template <bool WIDE, bool TH, bool RG, bool ENS, int KN2 = 0, int KTJ = 0, bool TAB = false>
__global__ void __maxnreg__(kMarchRegs)
    rk2_stage_march_f32c(RealStageParams p_in, MarchGeom g, EnsMarch em) {
    static_assert((KN2 == 0) == (KTJ == 0), "fixed geometry: both KN2 and KTJ");
    static_assert(!(TAB && (TH || ENS)), "TAB: the staged-table source of a single lattice");
    RealStageParams p = p_in;
    if constexpr (ENS) p.step = em.step + (em.ctr ? *em.ctr + (unsigned long long)em.offset : 0ull);
    else resolve_schedule(p);
    if constexpr (RG) reset_next_range(p);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
    float* s_tab = reinterpret_cast<float*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + g.tab_bytes);
    uint64_t* empty = full + 8;
    unsigned char* ring = smem + g.tab_bytes + 128;

    const int n0 = p.n0, n1 = p.n1, n2 = KN2 ? KN2 : p.n2;
    const int pitch = KN2 ? KN2 : g.pitch;
    const int TJ = KTJ ? KTJ : g.TJ;
    const uint32_t NS = (uint32_t)g.S;
    const int rows = TJ + 2;
    const int tpr = n2 >> 2;
    const int nc = TJ * tpr;
    const int t = threadIdx.x;

    if (t == 0) {
        for (uint32_t s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], nc / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if constexpr (TAB) stage_table_pairs(p, reinterpret_cast<float2*>(s_tab));  // (value, slope)
    else if (p.table_in_smem) stage_table<float>(p, s_tab);  // ends with __syncthreads
    else __syncthreads();

    // one [rows][pitch] block (bytes); a stage holds four
    const size_t plane_blk = KN2 ? (size_t)(KTJ + 2) * KN2 * 4 : (size_t)(g.stage_bytes >> 2);
    const size_t stage_b = 4 * plane_blk;
    // stage -> field f (0 phi, 1 pi) -> component c (0 hi, 1 lo)
    auto blk = [&](uint32_t stage, int f, int c) -> float* {
        return reinterpret_cast<float*>(ring + (size_t)stage * stage_b +
                                        (size_t)(2 * f + c) * plane_blk);
    };

    // ------------------------------------------------------------ producer
    if (t >= nc) {
        if (t != nc) return;
        const uint32_t plane_tx = (uint32_t)(4 * rows * n2 * 4);
        const float* const src_phi = static_cast<const float*>(p.phi);
        const float* const src_pi = static_cast<const float*>(p.pi);
        // test of the bounded waits: block 0 stops issuing at this ring position
        const uint32_t stop_at = (p.test_withhold > 0 && blockIdx.x == 0)
                                     ? (uint32_t)(p.test_withhold - 1) : 0xFFFFFFFFu;
        RingPos w{0, 0};
        uint32_t issued = 0;
        bool ok = true;
        const int64_t plane_n = (int64_t)n0 * n1 * n2;
        int n_items = g.items;
        if constexpr (ENS) {
            if (em.n_rids) n_items = min(g.items, *em.n_rids * em.items_per_rep);
        }
        BalRun br(g, p, blockIdx.x, gridDim.x);
        for (int item = blockIdx.x; ((!ENS && g.bal) ? br.more() : item < n_items) && ok;
             item += gridDim.x) {
            int it = item;
            const float *phi_hi = src_phi, *phi_lo = src_phi + plane_n;
            const float *pi_hi = src_pi, *pi_lo = src_pi + plane_n;
            if constexpr (ENS) {
                const int rl = item / em.items_per_rep;
                const int rid = em.rids[rl];
                if (!em.active[rid]) continue;
                it = item - rl * em.items_per_rep;
                const int64_t off = em.reps[rid].offset;
                if (off & 3) {  // bulk-copy sources must be 16-byte aligned: skipped
                    atomicExch(&g_device_status, (int)TIPT_ERR_ALIGN);
                    continue;
                }
                phi_hi = src_phi + off;
                phi_lo = src_phi + em.n_total + off;
                pi_hi = src_pi + off;
                pi_lo = src_pi + em.n_total + off;
            }
            int j0, i0, ni;
            if (!ENS && g.bal) {
                br.next(j0, i0, ni);
                j0 *= TJ;
            } else {
                const int ic = it / g.nJB;
                j0 = (it - ic * g.nJB) * TJ;
                i0 = p.i_begin + ic * g.CI;
                ni = min(g.CI, p.i_end - i0);
            }
            const int npl = ni + 2;
            for (int q = 0; q < npl; ++q) {
                if (issued == stop_at) {  // nothing is issued from here on
                    ok = false;
                    break;
                }
                if (issued >= NS && !mbar_wait(&empty[w.stage], w.phase ^ 1u)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&full[w.stage], plane_tx);
                int iw = i0 - 1 + q;
                iw = iw < 0 ? iw + n0 : (iw >= n0 ? iw - n0 : iw);
                // plane iw of the hi and lo planes of each field
                copy_tile_rows(blk(w.stage, 0, 0), phi_hi, iw, j0, rows, n1, n2, pitch, &full[w.stage]);
                copy_tile_rows(blk(w.stage, 0, 1), phi_lo, iw, j0, rows, n1, n2, pitch, &full[w.stage]);
                copy_tile_rows(blk(w.stage, 1, 0), pi_hi, iw, j0, rows, n1, n2, pitch, &full[w.stage]);
                copy_tile_rows(blk(w.stage, 1, 1), pi_lo, iw, j0, rows, n1, n2, pitch, &full[w.stage]);
                ++issued;
                w.next(NS);
            }
        }
        if (!ok && issued != stop_at) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
        RingPos d = w;
        for (uint32_t k = 0; k < NS && k < issued; ++k) {
            d.stage = d.stage == 0 ? NS - 1 : d.stage - 1;
            if (d.stage == NS - 1) d.phase ^= 1u;
            (void)mbar_wait(&full[d.stage], d.phase);
        }
        return;
    }

    // ----------------------------------------------------------- consumers
    const int lane = t & 31;
    const int r = 1 + t / tpr;                 // own tile row (1..TJ)
    const int k0 = 4 * (t - (r - 1) * tpr);    // first of the four own columns
    const int kml = k0 == 0 ? n2 - 1 : k0 - 1;
    const int kpr = k0 + 4 == n2 ? 0 : k0 + 4;
    F32CConst kc = f32c_const(p);
    float* phi_out = static_cast<float*>(p.phi_out);
    float* pi_out = static_cast<float*>(p.pi_out);
    // lo planes N sites after the hi planes (the lattice's, or the packed buffer's)
    int64_t N = (int64_t)n0 * n1 * n2;
    if constexpr (ENS) N = em.n_total;
    const int orow = r * pitch, urow = (r - 1) * pitch, drow = (r + 1) * pitch;
    // the batched replicas' own polynomial, amplitude and seed (set per item)
    float2 ec1 = make_float2(0.0f, 0.0f), ec2 = ec1, ec3 = ec1;
    bool ehas_c2 = false;
    uint64_t eseed = 0;

    RangeAcc racc;
    RingPos pm{0, 0};
    int n_items = g.items;  // the producer reads the same count
    if constexpr (ENS) {
        if (em.n_rids) n_items = min(g.items, *em.n_rids * em.items_per_rep);
    }
    BalRun br(g, p, blockIdx.x, gridDim.x);  // the producer's sequence of runs
    for (int item = blockIdx.x; (!ENS && g.bal) ? br.more() : item < n_items; item += gridDim.x) {
        int it = item;
        if constexpr (ENS) {
            const int rl = item / em.items_per_rep;
            const int rid = em.rids[rl];
            if (!em.active[rid]) continue;
            it = item - rl * em.items_per_rep;
            const tipt_replica& rp = em.reps[rid];
            if (rp.offset & 3) continue;  // skipped by the producer too
            phi_out = static_cast<float*>(p.phi_out) + rp.offset;
            pi_out = static_cast<float*>(p.pi_out) + rp.offset;
            const float f1 = (float)rp.c1, f2 = (float)rp.c2, f3 = (float)rp.c3;
            ec1 = make_float2(f1, f1);
            ec2 = make_float2(f2, f2);
            ec3 = make_float2(f3, f3);
            ehas_c2 = rp.c2 != 0.0;
            kc.ns = (float)rp.noise_scale;
            eseed = rp.seed;
        }
        int j0, i0, ni;
        if (!ENS && g.bal) {
            br.next(j0, i0, ni);
            j0 *= TJ;
        } else {
            const int ic = it / g.nJB;
            j0 = (it - ic * g.nJB) * TJ;
            i0 = p.i_begin + ic * g.CI;
            ni = min(g.CI, p.i_end - i0);
        }
        const int jw = j0 + r - 1;
        RingPos pc = pm, pp;
        pc.next(NS);
        pp = pc;
        pp.next(NS);
        if (!mbar_wait(&full[pm.stage], pm.phase) || !mbar_wait(&full[pc.stage], pc.phase)) {
            if (lane == 0) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
            return;
        }
        for (int q = 0; q < ni; ++q) {
            const int i = i0 + q;
            const int64_t rowoff = ((int64_t)i * n1 + jw) * n2 + k0;
            // the noise reads no tile: drawn before the wait for the next plane
            float2 kick[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint64_t site;
                if constexpr (WIDE) site = (uint64_t)(rowoff + p.site_offset + 2 * h);
                else site = (uint32_t)(rowoff + p.site_offset) + (uint32_t)(2 * h);
                if constexpr (ENS) {
                    // the replica's own seed and amplitude (site_kick_f32c2's hash branch)
                    kick[h] = kc.ns == 0.0f ? make_float2(0.0f, 0.0f)
                                            : v_mul(vs<float2>(kc.ns),
                                                    gauss_cos_f2(noise_key(site, p.step, p.mul, eseed),
                                                                 noise_key(site + 1, p.step, p.mul, eseed)));
                } else if constexpr (TAB) {
                    // hash noise: site_kick_f32c2's hash branch
                    kick[h] = p.ns_eff == 0.0 ? make_float2(0.0f, 0.0f)
                                              : v_mul(vs<float2>(kc.ns),
                                                      gauss_cos_f2(noise_key(site, p.step, p.mul, p.seed),
                                                                   noise_key(site + 1, p.step, p.mul, p.seed)));
                } else {
                    kick[h] = site_kick_f32c2(p, kc, site);
                }
            }
            // the centre plane is resident: its values and V' at the centre and
            // the midpoint are evaluated before the wait as well
            F32CPre<float2> pre[2];
            float4 cen[2][2];  // [field][hi, lo], kept for the stencil after the wait
#pragma unroll
            for (int f = 0; f < 2; ++f)
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    cen[f][c] = *reinterpret_cast<const float4*>(blk(pc.stage, f, c) + orow + k0);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const auto pick = [h](const float4& v) {
                    return h ? make_float2(v.z, v.w) : make_float2(v.x, v.y);
                };
                if constexpr (ENS)
                    pre[h] = pre_f32c_vp<float2>(p, pick(cen[0][0]), pick(cen[0][1]), pick(cen[1][0]),
                                                 pick(cen[1][1]), [&](float2 x) {
                                                     return poly_vprime_v<float2>(ec1, ec2, ec3, ehas_c2, x);
                                                 });
                else if constexpr (TAB)  // the V' row staged in shared memory: vprime_v's branch
                    pre[h] = pre_f32c_vp<float2>(p, pick(cen[0][0]), pick(cen[0][1]), pick(cen[1][0]),
                                                 pick(cen[1][1]), [&](float2 x) {
                                                     return lerp_pairs_f32<float2>(
                                                         reinterpret_cast<const float2*>(s_tab),
                                                         v_fma(x, p.k2.dinv, p.k2.tmd), kc.last);
                                                 });
                else
                    pre[h] = pre_f32c<float2, TH>(p, kc, s_tab, pick(cen[0][0]), pick(cen[0][1]),
                                                  pick(cen[1][0]), pick(cen[1][1]));
            }
            if (!mbar_wait(&full[pp.stage], pp.phase)) {
                if (lane == 0) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
                return;
            }
            F32CIn<float2> in[2];
#pragma unroll
            for (int f = 0; f < 2; ++f) {
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const float* sc = blk(pc.stage, f, c);
                    const float4 ce = cen[f][c];
                    const float4 jm = *reinterpret_cast<const float4*>(sc + urow + k0);
                    const float4 jp = *reinterpret_cast<const float4*>(sc + drow + k0);
                    const float4 im = *reinterpret_cast<const float4*>(blk(pm.stage, f, c) + orow + k0);
                    const float4 ip = *reinterpret_cast<const float4*>(blk(pp.stage, f, c) + orow + k0);
                    // k-1 of site 0 and k+1 of site 3 (scalar reads: fewer instructions
                    // than lane shuffles, which this issue-bound kernel prefers to the
                    // 4-way bank conflict they remove)
                    const float kl = sc[orow + kml], kr = sc[orow + kpr];
                    // site pairs (0,1) and (2,3): centre and the i and j neighbours
                    const float2 cc[2] = {make_float2(ce.x, ce.y), make_float2(ce.z, ce.w)};
                    const float2 nb[2][4] = {
                        {make_float2(ip.x, ip.y), make_float2(im.x, im.y), make_float2(jp.x, jp.y),
                         make_float2(jm.x, jm.y)},
                        {make_float2(ip.z, ip.w), make_float2(im.z, im.w), make_float2(jp.z, jp.w),
                         make_float2(jm.z, jm.w)}};
                    // the four sites' values with their k neighbours: v[1..4] own, v[0], v[5]
                    const float v[6] = {kl, ce.x, ce.y, ce.z, ce.w, kr};
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        // lanes: sites 2h, 2h+1 (v indices 2h+1, 2h+2); the k pair of a
                        // site is formed in its own lane (order of stencil_sums_k)
                        const int a = 2 * h + 1, b = 2 * h + 2;
                        float2 acc;
                        if (c == 0) {  // dh = sum (hi_n - hi_c)
                            acc = v_add(v_sub(nb[h][0], cc[h]), v_sub(nb[h][1], cc[h]));
                            acc = v_add(acc, v_sub(nb[h][2], cc[h]));
                            acc = v_add(acc, v_sub(nb[h][3], cc[h]));
                            const float2 kk = make_float2(
                                __fadd_rn(__fsub_rn(v[a + 1], v[a]), __fsub_rn(v[a - 1], v[a])),
                                __fadd_rn(__fsub_rn(v[b + 1], v[b]), __fsub_rn(v[b - 1], v[b])));
                            acc = v_add(acc, kk);
                        } else {       // dl = fma(-6, lo_c, sum lo_n)
                            acc = v_add(v_add(v_add(nb[h][0], nb[h][1]), nb[h][2]), nb[h][3]);
                            const float2 kk = make_float2(__fadd_rn(v[a + 1], v[a - 1]),
                                                          __fadd_rn(v[b + 1], v[b - 1]));
                            acc = v_fma(vs<float2>(-6.0f), cc[h], v_add(acc, kk));
                        }
                        if (f == 0) {
                            if (c == 0) { in[h].dh_phi = acc; in[h].phh = cc[h]; }
                            else { in[h].dl_phi = acc; in[h].phl = cc[h]; }
                        } else {
                            if (c == 0) { in[h].dh_pi = acc; in[h].pih = cc[h]; }
                            else { in[h].dl_pi = acc; in[h].pil = cc[h]; }
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[pm.stage]);  // plane i-1 is no longer read
            float2 o[2][4];
#pragma unroll
            for (int h = 0; h < 2; ++h)
                post_f32c<float2>(p, in[h], pre[h], kick[h], o[h][0], o[h][1], o[h][2], o[h][3]);
            *reinterpret_cast<float4*>(phi_out + rowoff) = make_float4(o[0][0].x, o[0][0].y, o[1][0].x, o[1][0].y);
            *reinterpret_cast<float4*>(phi_out + N + rowoff) = make_float4(o[0][1].x, o[0][1].y, o[1][1].x, o[1][1].y);
            *reinterpret_cast<float4*>(pi_out + rowoff) = make_float4(o[0][2].x, o[0][2].y, o[1][2].x, o[1][2].y);
            *reinterpret_cast<float4*>(pi_out + N + rowoff) = make_float4(o[0][3].x, o[0][3].y, o[1][3].x, o[1][3].y);
            if constexpr (RG) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    racc.fold_ff(o[h][0].x, o[h][1].x);
                    racc.fold_ff(o[h][0].y, o[h][1].y);
                }
            }
            pm = pc;
            pc = pp;
            pp.next(NS);
        }
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&empty[pm.stage]);
            mbar_arrive(&empty[pc.stage]);
        }
        pm = pp;
    }
    if constexpr (RG) racc.flush(p.range);
}

// ------------------------------- alternative integrators, F32C marching ----
// Overdamped Euler-Maruyama and the two BAOAB passes (R:2115, R:1974; complex
// C:2422, C:2223) on the marching ring: the stencil reads the field alone, so
// a ring stage holds the hi and lo planes of phi (real) or of phi1 and phi2
// (complex); pi (the BAOAB passes) is read and written at the thread's own
// four sites.  The per-component arithmetic is alt_real_site_f32c and the
// complex force complex_force_v, which the generic kernels run too, so both
// give the same bits.
// SRC: kCsrcAny dispatches on the V' source at run time; kCsrcTab (and, for the
// complex force, kCsrcTabEps) fix the staged table at compile time.
// KN2, KTJ > 0: rows of KN2 sites in KTJ-row tiles fixed at compile time (as
// the RK2 stage's fixed geometry).
template <int MODE, bool CPLX, bool WIDE, int SRC = kCsrcAny, int KN2 = 0, int KTJ = 0>
__global__ void __maxnreg__(kMarchRegs) alt_march_f32c(AltParams p, MarchGeom g) {
    constexpr int NF = CPLX ? 2 : 1;  // stencil fields
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
    float* s_tab = reinterpret_cast<float*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + g.tab_bytes);
    uint64_t* empty = full + 8;
    unsigned char* ring = smem + g.tab_bytes + 128;

    const int n0 = p.n0, n1 = p.n1, n2 = KN2 ? KN2 : p.n2;
    const int pitch = KN2 ? KN2 : g.pitch;
    const int TJ = KTJ ? KTJ : g.TJ;
    const uint32_t NS = (uint32_t)g.S;
    const int rows = TJ + 2;
    const int tpr = n2 >> 2;
    const int nc = TJ * tpr;
    const int t = threadIdx.x;

    if (t == 0) {
        for (uint32_t s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], nc / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (p.v.table_in_smem)
        for (int q = t; q < p.v.npts; q += blockDim.x) s_tab[q] = (float)__ldg(p.v.table + q);
    __syncthreads();

    // one [rows][pitch] block (bytes); a stage holds 2 NF
    const size_t plane_blk =
        KN2 ? (size_t)(KTJ + 2) * KN2 * 4 : (size_t)(g.stage_bytes / (2 * NF));
    const size_t stage_b = KN2 ? 2 * NF * plane_blk : (size_t)g.stage_bytes;
    auto blk = [&](uint32_t stage, int f, int c) -> float* {     // field f, c: 0 hi, 1 lo
        return reinterpret_cast<float*>(ring + (size_t)stage * stage_b +
                                        (size_t)(2 * f + c) * plane_blk);
    };

    // ------------------------------------------------------------ producer
    if (t >= nc) {
        if (t != nc) return;
        const uint32_t plane_tx = (uint32_t)(2 * NF * rows * n2 * 4);
        RingPos w{0, 0};
        uint32_t issued = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < g.items && ok; item += gridDim.x) {
            const int ic = item / g.nJB;
            const int j0 = (item - ic * g.nJB) * TJ, i0 = ic * g.CI;
            const int npl = min(g.CI, n0 - i0) + 2;
            for (int q = 0; q < npl; ++q) {
                if (issued >= NS && !mbar_wait(&empty[w.stage], w.phase ^ 1u)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&full[w.stage], plane_tx);
                int iw = i0 - 1 + q;
                iw = iw < 0 ? iw + n0 : (iw >= n0 ? iw - n0 : iw);
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    const float* src = static_cast<const float*>(p.f[f]);
                    copy_tile_rows(blk(w.stage, f, 0), src, iw, j0, rows, n1, n2, pitch, &full[w.stage]);
                    copy_tile_rows(blk(w.stage, f, 1), src, n0 + iw, j0, rows, n1, n2, pitch,
                                   &full[w.stage]);
                }
                ++issued;
                w.next(NS);
            }
        }
        if (!ok) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
        RingPos d = w;
        for (uint32_t k = 0; k < NS && k < issued; ++k) {
            d.stage = d.stage == 0 ? NS - 1 : d.stage - 1;
            if (d.stage == NS - 1) d.phase ^= 1u;
            (void)mbar_wait(&full[d.stage], d.phase);
        }
        return;
    }

    // ----------------------------------------------------------- consumers
    const int lane = t & 31;
    const int r = 1 + t / tpr;
    const int k0 = 4 * (t - (r - 1) * tpr);
    const int kml = k0 == 0 ? n2 - 1 : k0 - 1;
    const int kpr = k0 + 4 == n2 ? 0 : k0 + 4;
    const int64_t N = (int64_t)n0 * n1 * n2;
    const int orow = r * pitch, urow = (r - 1) * pitch, drow = (r + 1) * pitch;
    const bool noisy = (MODE == kOD && p.ns != 0.0) || (MODE == kBA1 && p.c2 != 0.0);
    const float tminf = (float)p.v.tmin, dinvf = (float)p.v.dinv, last = (float)(p.v.npts - 2);

    RingPos pm{0, 0};
    for (int item = blockIdx.x; item < g.items; item += gridDim.x) {
        const int ic = item / g.nJB;
        const int j0 = (item - ic * g.nJB) * TJ, i0 = ic * g.CI;
        const int ni = min(g.CI, n0 - i0);
        const int jw = j0 + r - 1;
        RingPos pc = pm, pp;
        pc.next(NS);
        pp = pc;
        pp.next(NS);
        if (!mbar_wait(&full[pm.stage], pm.phase) || !mbar_wait(&full[pc.stage], pc.phase)) {
            if (lane == 0) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
            return;
        }
        for (int q = 0; q < ni; ++q) {
            const int64_t rowoff = ((int64_t)(i0 + q) * n1 + jw) * n2 + k0;
            // pi at the thread's own four sites (BAOAB passes), loaded before the
            // noise so the loads are in flight during it, the wait and the stencil
            // (the complex first pass, short of registers there, loads after the stencil)
            constexpr bool kPiEarly = !(CPLX && MODE == kBA1);
            float4 piv[NF][2];  // [field][hi, lo]
            const auto load_pi = [&]() {
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    const float* pif = static_cast<const float*>(p.f[NF + f]);
                    piv[f][0] = *reinterpret_cast<const float4*>(pif + rowoff);
                    piv[f][1] = *reinterpret_cast<const float4*>(pif + N + rowoff);
                }
            };
            if constexpr (MODE != kOD && kPiEarly) load_pi();
            // the noise reads no tile: drawn before the wait for the next plane
            float2 zz[2][NF];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint64_t site;
                if constexpr (WIDE) site = (uint64_t)(rowoff + 2 * h);
                else site = (uint32_t)rowoff + (uint32_t)(2 * h);
                const uint64_t ka = noise_key(site, p.step, kPass2Mul, p.seed);
                const uint64_t kb = noise_key(site + 1, p.step, kPass2Mul, p.seed);
#pragma unroll
                for (int f = 0; f < NF; ++f) zz[h][f] = make_float2(0.0f, 0.0f);
                if constexpr (CPLX) {
                    if (noisy) gauss_pair_f2(ka, kb, zz[h][0], zz[h][1]);
                } else {
                    if (noisy) zz[h][0] = gauss_cos_f2(ka, kb);
                }
            }
            if (!mbar_wait(&full[pp.stage], pp.phase)) {
                if (lane == 0) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
                return;
            }
            float2 dsum[2][NF][2], cen[2][NF][2];  // [pair][field][hi, lo]
#pragma unroll
            for (int f = 0; f < NF; ++f) {
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const float* sc = blk(pc.stage, f, c);
                    const float4 ce = *reinterpret_cast<const float4*>(sc + orow + k0);
                    const float4 jm = *reinterpret_cast<const float4*>(sc + urow + k0);
                    const float4 jp = *reinterpret_cast<const float4*>(sc + drow + k0);
                    const float4 im = *reinterpret_cast<const float4*>(blk(pm.stage, f, c) + orow + k0);
                    const float4 ip = *reinterpret_cast<const float4*>(blk(pp.stage, f, c) + orow + k0);
                    float kl = __shfl_up_sync(0xffffffffu, ce.w, 1);
                    float kr = __shfl_down_sync(0xffffffffu, ce.x, 1);
                    if (lane == 0 || k0 == 0) kl = sc[orow + kml];
                    if (lane == 31 || k0 + 4 == n2) kr = sc[orow + kpr];
                    const float2 cc[2] = {make_float2(ce.x, ce.y), make_float2(ce.z, ce.w)};
                    const float2 nb[2][6] = {
                        {make_float2(ip.x, ip.y), make_float2(im.x, im.y), make_float2(jp.x, jp.y),
                         make_float2(jm.x, jm.y), make_float2(ce.y, ce.z), make_float2(kl, ce.x)},
                        {make_float2(ip.z, ip.w), make_float2(im.z, im.w), make_float2(jp.z, jp.w),
                         make_float2(jm.z, jm.w), make_float2(ce.w, kr), make_float2(ce.y, ce.z)}};
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        float2 acc;
                        if (c == 0) {  // dh = sum (hi_n - hi_c)
                            acc = v_sub(nb[h][0], cc[h]);
#pragma unroll
                            for (int n = 1; n < 6; ++n) acc = v_add(acc, v_sub(nb[h][n], cc[h]));
                        } else {       // dl = fma(-6, lo_c, sum lo_n)
                            acc = nb[h][0];
#pragma unroll
                            for (int n = 1; n < 6; ++n) acc = v_add(acc, nb[h][n]);
                            acc = v_fma(vs<float2>(-6.0f), cc[h], acc);
                        }
                        dsum[h][f][c] = acc;
                        cen[h][f][c] = cc[h];
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[pm.stage]);  // plane i-1 is no longer read
            if constexpr (MODE != kOD && !kPiEarly) load_pi();
            float ah[NF][4], al[NF][4], bh[NF][4], bl[NF][4];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float2* z = zz[h];
                float2 vp[NF];
                if constexpr (CPLX) {
                    complex_force_v<float2, SRC>(p.v, s_tab, tminf, dinvf,
                                            v_add(cen[h][0][0], cen[h][0][1]),
                                            v_add(cen[h][1][0], cen[h][1][1]), vp[0], vp[1]);
                } else {
                    const float2 x = v_add(cen[h][0][0], cen[h][0][1]);
                    if (SRC == kCsrcAny && p.v.vkind == TIPT_VP_POLY) {
                        const float2 d = v_fma(v_mul(v_mul(vs<float2>((float)p.v.c3), x), x), x,
                                               v_mul(vs<float2>((float)p.v.c1), x));
                        vp[0] = p.v.c2 != 0.0 ? v_fma(v_mul(vs<float2>((float)p.v.c2), x), x, d) : d;
                    } else {
                        vp[0] = lerp_table_f32<float2>(
                            s_tab, v_mul(v_sub(x, vs<float2>(tminf)), vs<float2>(dinvf)), last);
                    }
                }
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    float vh[2] = {0.0f, 0.0f}, vl[2] = {0.0f, 0.0f};
                    if constexpr (MODE != kOD) {
                        const float4 a = piv[f][0], b = piv[f][1];
                        vh[0] = h ? a.z : a.x; vh[1] = h ? a.w : a.y;
                        vl[0] = h ? b.z : b.x; vl[1] = h ? b.w : b.y;
                    }
                    alt_real_site_f32c<MODE>(p, cen[h][f][0].x, cen[h][f][1].x, dsum[h][f][0].x,
                                             dsum[h][f][1].x, vp[f].x, z[f].x, vh[0], vl[0],
                                             ah[f][2 * h], al[f][2 * h], bh[f][2 * h], bl[f][2 * h]);
                    alt_real_site_f32c<MODE>(p, cen[h][f][0].y, cen[h][f][1].y, dsum[h][f][0].y,
                                             dsum[h][f][1].y, vp[f].y, z[f].y, vh[1], vl[1],
                                             ah[f][2 * h + 1], al[f][2 * h + 1], bh[f][2 * h + 1],
                                             bl[f][2 * h + 1]);
                }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                if constexpr (MODE != kBA2) {
                    float* o = static_cast<float*>(p.o[f]);
                    *reinterpret_cast<float4*>(o + rowoff) = make_float4(ah[f][0], ah[f][1], ah[f][2], ah[f][3]);
                    *reinterpret_cast<float4*>(o + N + rowoff) = make_float4(al[f][0], al[f][1], al[f][2], al[f][3]);
                }
                if constexpr (MODE != kOD) {
                    float* o = static_cast<float*>(p.o[NF + f]);
                    *reinterpret_cast<float4*>(o + rowoff) = make_float4(bh[f][0], bh[f][1], bh[f][2], bh[f][3]);
                    *reinterpret_cast<float4*>(o + N + rowoff) = make_float4(bl[f][0], bl[f][1], bl[f][2], bl[f][3]);
                }
            }
            pm = pc;
            pc = pp;
            pp.next(NS);
        }
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&empty[pm.stage]);
            mbar_arrive(&empty[pc.stage]);
        }
        pm = pp;
    }
}

// ----------------------------------------------------- complex, F32C ----
// Complex field in compensated FP32: four planar fields (phi1, phi2, pi1, pi2;
// hi plane then lo plane each), so a ring stage holds eight (TJ+2)-row blocks.
// A consumer thread owns two consecutive sites of its row (one 8-byte vector
// per plane and neighbour) and evaluates them in the two lanes of the packed
// FP32x2 instructions with the arithmetic of the generic kernel
// (complex_update_f32c), so the results are bitwise identical.
//
// KKS, KTJ > 0: segments of KKS sites (pitch KKS) in KTJ-row tiles fixed at
// compile time, as the real stage's fixed geometry (the launcher takes it when
// the run-time geometry is exactly that one).
template <bool WIDE, bool RG, int KKS = 0, int KTJ = 0>
__global__ void __maxnreg__(kMarchRegs)
    complex_stage_march_f32c(const __grid_constant__ CUtensorMap tm0,
                             const __grid_constant__ CUtensorMap tm1,
                             const __grid_constant__ CUtensorMap tm2,
                             const __grid_constant__ CUtensorMap tm3, ComplexStageParams p,
                             MarchGeom g) {
    static_assert((KKS == 0) == (KTJ == 0) && KKS % 32 == 0, "fixed geometry: KKS and KTJ");
    if constexpr (RG) reset_range_words(p.range_next);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
    float* s_tab = reinterpret_cast<float*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + g.tab_bytes);
    uint64_t* empty = full + 8;
    unsigned char* ring = smem + g.tab_bytes + 128;

    const int n0 = p.n0, n1 = p.n1, n2 = p.n2;
    const int pitch = KKS ? KKS : g.pitch;
    const int TJ = KTJ ? KTJ : g.TJ;
    const uint32_t NS = (uint32_t)g.S;
    const int rows = TJ + 2;
    const int KS = KKS ? KKS : g.KS;
    const bool split = g.nKS > 1;
    const int tpr = KS >> 1;
    const int nc = TJ * tpr;
    const int t = threadIdx.x;
    const int nJK = g.nJB * g.nKS;

    if (t == 0) {
        for (uint32_t s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], nc / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (p.table_in_smem)
        for (int q = t; q < p.npts; q += blockDim.x) s_tab[q] = (float)__ldg(p.table + q);
    __syncthreads();

    // one [rows][pitch] block, bytes; a stage holds eight
    const size_t plane_blk = KKS ? (size_t)(KTJ + 2) * KKS * 4 : (size_t)((g.halo_off) >> 3);
    const size_t stage_b = KKS ? 8 * plane_blk : (size_t)g.stage_bytes;
    // stage -> field f (phi1, phi2, pi1, pi2) -> component c (0 hi, 1 lo)
    auto blk = [&](uint32_t stage, int f, int c) -> float* {
        return reinterpret_cast<float*>(ring + (size_t)stage * stage_b +
                                        (size_t)(2 * f + c) * plane_blk);
    };
    // split rows: the k-1 neighbour of a segment's first site and the k+1 neighbour of its
    // last site are copied from global memory by the two edge threads of each tile row
    // (cp.async, one plane ahead) into a per-thread double buffer after the ring:
    // [TJ rows][2 sides][2 slots][8 = field x component]
    float* halo = reinterpret_cast<float*>(ring + (size_t)NS * stage_b);

    // ------------------------------------------------------------ producer
    if (t >= nc) {
        if (t != nc) return;
        const CUtensorMap* tm[4] = {&tm0, &tm1, &tm2, &tm3};
        const uint32_t plane_tx = (uint32_t)(8 * rows * KS * 4);
        RingPos w{0, 0};
        uint32_t issued = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < g.items && ok; item += gridDim.x) {
            const int ic = item / nJK;
            const int jk = item - ic * nJK;
            const int jb = jk / g.nKS;
            const int k0s = (jk - jb * g.nKS) * KS;
            const int j0 = jb * TJ, i0 = ic * g.CI;
            const int npl = min(g.CI, n0 - i0) + 2;
            for (int q = 0; q < npl; ++q) {
                if (issued >= NS && !mbar_wait(&empty[w.stage], w.phase ^ 1u)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&full[w.stage], plane_tx);
                int iw = i0 - 1 + q;
                iw = iw < 0 ? iw + n0 : (iw >= n0 ? iw - n0 : iw);
                for (int rr = 0; rr < rows; ++rr) {
                    int jr = j0 - 1 + rr;
                    jr = jr < 0 ? jr + n1 : (jr >= n1 ? jr - n1 : jr);
                    for (int kb = 0; kb < KS; kb += g.BK) {
                        const int o = rr * pitch + kb;
#pragma unroll
                        for (int f = 0; f < 4; ++f) {
                            // plane iw = hi, plane n0 + iw = lo
                            tma_row(blk(w.stage, f, 0) + o, tm[f], k0s + kb, jr, iw, &full[w.stage]);
                            tma_row(blk(w.stage, f, 1) + o, tm[f], k0s + kb, jr, n0 + iw,
                                    &full[w.stage]);
                        }
                    }
                }
                ++issued;
                w.next(NS);
            }
        }
        if (!ok) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
        RingPos d = w;
        for (uint32_t k = 0; k < NS && k < issued; ++k) {
            d.stage = d.stage == 0 ? NS - 1 : d.stage - 1;
            if (d.stage == NS - 1) d.phase ^= 1u;
            (void)mbar_wait(&full[d.stage], d.phase);
        }
        return;
    }

    // ----------------------------------------------------------- consumers
    const int lane = t & 31;
    const int r = 1 + t / tpr;                 // own tile row (1..TJ)
    const int k0 = 2 * (t - (r - 1) * tpr);    // first of the two own columns (in the segment)
    const bool edge_l = k0 == 0, edge_r = k0 + 2 == KS;
    const int kml = edge_l ? KS - 1 : k0 - 1;  // unsplit rows wrap inside the row
    const int kpr = edge_r ? 0 : k0 + 2;
    const float tminf = (float)p.tmin, dinvf = (float)p.dinv;
    const int64_t N = (int64_t)n0 * n1 * n2;
    const int orow = r * pitch, urow = (r - 1) * pitch, drow = (r + 1) * pitch;
    auto force = [&](float2 q1, float2 q2, int, float2& d1, float2& d2) {
        complex_force_v<float2>(p, s_tab, tminf, dinvf, q1, q2, d1, d2);
    };
    const bool edge = split && (edge_l || edge_r);
    float* my_halo = halo + ((r - 1) * 2 + (edge_r ? 1 : 0)) * 16;
    // issue the copies of plane i's 8 halo values (row jw, column kcol) into slot
    auto fetch_halo = [&](int i, int jw, int kcol, int slot) {
        const int64_t off = ((int64_t)i * n1 + jw) * n2 + kcol;
#pragma unroll
        for (int f = 0; f < 4; ++f)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const float* src = static_cast<const float*>(p.f[f]) + (c ? N : 0) + off;
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                                 smem_addr(my_halo + slot * 8 + 2 * f + c)),
                             "l"(src)
                             : "memory");
            }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    RangeAcc racc;
    RingPos pm{0, 0};
    for (int item = blockIdx.x; item < g.items; item += gridDim.x) {
        const int ic = item / nJK;
        const int jk = item - ic * nJK;
        const int jb = jk / g.nKS;
        const int k0s = (jk - jb * g.nKS) * KS;
        const int j0 = jb * TJ, i0 = ic * g.CI;
        const int ni = min(g.CI, n0 - i0);
        const int jw = j0 + r - 1;
        RingPos pc = pm, pp;
        pc.next(NS);
        pp = pc;
        pp.next(NS);
        const int kcol = edge_l ? (k0s - 1 + n2) % n2 : (k0s + KS) % n2;
        if (edge) fetch_halo(i0, jw, kcol, 0);
        if (!mbar_wait(&full[pm.stage], pm.phase) || !mbar_wait(&full[pc.stage], pc.phase)) {
            if (lane == 0) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
            if (edge) asm volatile("cp.async.wait_all;" ::: "memory");
            return;
        }
        for (int q = 0; q < ni; ++q) {
            const int i = i0 + q;
            const int64_t rowoff = ((int64_t)i * n1 + jw) * n2 + k0s + k0;
            // the noise reads no tile: drawn before the wait for the next plane
            float2 kick[2];
            if constexpr (WIDE)
                complex_kick_f32c2(p, (uint64_t)rowoff, (uint64_t)(rowoff + 1), kick[0], kick[1]);
            else
                complex_kick_f32c2(p, (uint32_t)rowoff, (uint32_t)rowoff + 1u, kick[0], kick[1]);
            if (!mbar_wait(&full[pp.stage], pp.phase)) {
                if (lane == 0) atomicExch(&g_device_status, (int)TIPT_ERR_TIMEOUT);
                if (edge) asm volatile("cp.async.wait_all;" ::: "memory");
                return;
            }
            float hv[8];
            if (edge) {
                asm volatile("cp.async.wait_all;" ::: "memory");
                const float* hs = my_halo + (q & 1) * 8;
#pragma unroll
                for (int e = 0; e < 8; ++e) hv[e] = hs[e];
                if (q + 1 < ni) fetch_halo(i + 1, jw, kcol, (q + 1) & 1);
            }
            CplxIn<float2> in;
#pragma unroll
            for (int f = 0; f < 4; ++f) {
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const float* sc = blk(pc.stage, f, c);
                    const float2 ce = *reinterpret_cast<const float2*>(sc + orow + k0);
                    const float2 jm = *reinterpret_cast<const float2*>(sc + urow + k0);
                    const float2 jp = *reinterpret_cast<const float2*>(sc + drow + k0);
                    const float2 im = *reinterpret_cast<const float2*>(blk(pm.stage, f, c) + orow + k0);
                    const float2 ip = *reinterpret_cast<const float2*>(blk(pp.stage, f, c) + orow + k0);
                    // k-1 / k+1 from the neighbouring lanes; at warp, row and segment
                    // ends from shared memory or the copied segment halo
                    float kl = __shfl_up_sync(0xffffffffu, ce.y, 1);
                    float kr = __shfl_down_sync(0xffffffffu, ce.x, 1);
                    if (lane == 0 || edge_l) kl = (split && edge_l) ? hv[2 * f + c] : sc[orow + kml];
                    if (lane == 31 || edge_r) kr = (split && edge_r) ? hv[2 * f + c] : sc[orow + kpr];
                    // lanes = sites k0, k0+1; the i and j neighbours in the order ip, im,
                    // jp, jm, then each site's k pair formed in its own lane (the order of
                    // stencil_sums_k)
                    float2 acc;
                    if (c == 0) {  // dh = sum (hi_n - hi_c)
                        acc = v_add(v_add(v_add(v_sub(ip, ce), v_sub(im, ce)), v_sub(jp, ce)),
                                    v_sub(jm, ce));
                        // k pairs from the neighbour differences em, e0, e1: km - c is
                        // -(the difference on the left) exactly, so (kp - c) + (km - c)
                        // rounds once as e_right - e_left (the same bits)
                        const float em = __fsub_rn(ce.x, kl), e0 = __fsub_rn(ce.y, ce.x),
                                    e1 = __fsub_rn(kr, ce.y);
                        const float2 kk = make_float2(__fsub_rn(e0, em), __fsub_rn(e1, e0));
                        in.dh[f] = v_add(acc, kk);
                        in.ch[f] = ce;
                    } else {       // dl = fma(-6, lo_c, sum lo_n)
                        acc = v_add(v_add(v_add(ip, im), jp), jm);
                        const float2 kk = make_float2(__fadd_rn(ce.y, kl), __fadd_rn(kr, ce.x));
                        in.dl[f] = v_fma(vs<float2>(-6.0f), ce, v_add(acc, kk));
                        in.cl[f] = ce;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[pm.stage]);  // plane i-1 is no longer read
            float2 oh[4], ol[4];
            complex_update_f32c<float2>(p, in, kick, force, oh, ol);
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                float* po = static_cast<float*>(p.o[f]);
                *reinterpret_cast<float2*>(po + rowoff) = oh[f];
                *reinterpret_cast<float2*>(po + N + rowoff) = ol[f];
            }
            if constexpr (RG) {
                fold_rho_ff(racc, oh[0].x, ol[0].x, oh[1].x, ol[1].x);
                fold_rho_ff(racc, oh[0].y, ol[0].y, oh[1].y, ol[1].y);
            }
            pm = pc;
            pc = pp;
            pp.next(NS);
        }
        __syncwarp();
        if (lane == 0) {
            mbar_arrive(&empty[pm.stage]);
            mbar_arrive(&empty[pc.stage]);
        }
        pm = pp;
    }
    if constexpr (RG) racc.flush(p.range);
}

// ------------------------------------------------------------------ host ---
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                              const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                              const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeFn encode_fn() {
    static EncodeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(f);
    }
    return fn;
}

// 3-D map of one field: (n2, n1, planes) with elements of `es` bytes (FP64
// fields: planes = n0; planar FP32 pairs: planes = 2*n0, hi then lo).
static bool make_map(CUtensorMap* tm, const void* base, int planes, int n1, int n2, int es,
                     int BK) {
    EncodeFn enc = encode_fn();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)n2, (cuuint64_t)n1, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)n2 * es, (cuuint64_t)n2 * es * n1};
    const cuuint32_t box[3] = {(cuuint32_t)BK, 1, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(tm, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
               const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tile shape; 0 = choose automatically.  Set by tipt_set_march_tiles().
static int g_force_tj = 0, g_force_ci = 0, g_force_stages = 0;
// Kernels compiled for a fixed geometry used where the run-time geometry is
// theirs (tipt_set_march_fixed(); on by default).
static bool g_fixed_geom = true;
// The compensated-FP32 stage's balanced split of the work (MarchGeom::bal).
static bool g_balance = true;

// One-shot test of the bounded waits (tipt_test_withhold_plane): the next
// compensated-FP32 marching stage launch withholds a ring position in block 0.
static int g_test_withhold = 0;

// TMA box width (elements of `es` bytes).  A tensor copy's shared-memory
// destination must be 128-byte aligned: rows sit at multiples of the
// 128-byte pitch, and a row split into several boxes needs box widths of a
// multiple of 128 bytes.
static int pick_bk(int n2, int es) {
    if (n2 <= 256) return n2;
    const int step = 128 / es;
    for (int bk = 256; bk >= step; bk -= step)
        if (n2 % bk == 0) return bk;
    return 0;
}

static int round128(int x) { return (x + 127) & ~127; }

constexpr int kSmemPerSm = 228 * 1024;   // B200 shared memory per SM
constexpr int kSmemPerCta = 227 * 1024;  // largest opt-in allocation per CTA
constexpr int kSmemReserve = 1024;       // per-CTA reservation of the runtime
constexpr int kWarpsPerSm = 18;          // at kMarchRegs registers per thread

static int64_t smem_need(const MarchGeom& g) {
    return 128 + (int64_t)g.tab_bytes + 128 + (int64_t)g.S * g.stage_bytes;  // + alignment slack
}

// CTAs per SM for a geometry (shared memory and register-file bound).
static int ctas_per_sm(const MarchGeom& g, int tpr) {
    const int64_t need = smem_need(g) + kSmemReserve;
    int by_smem = (int)(kSmemPerSm / need);
    const int warps = g.TJ * tpr / 32 + 1;
    int by_warps = kWarpsPerSm / warps;
    return by_smem < by_warps ? by_smem : by_warps;
}

// Shared-memory ring layout of a storage: FP64 -> one 8-byte plane per field;
// F32C -> two 4-byte planes (hi, lo) per field.
static int layout_es(int storage) { return storage == TIPT_F64 ? 8 : 4; }
static int layout_planes(int storage) { return storage == TIPT_F32C ? 2 : 1; }

// Tile geometry of the real-field marching kernels: n1 x n2 rows, nplanes
// planes to compute, `comps` component planes of `es`-byte elements per ring
// stage (RK2: phi and pi, hi and lo for F32C; the alternative integrators: phi).
static bool geometry_dims(int n1, int n2, int nplanes, int es, int comps, int64_t smem_table,
                          MarchGeom& g, int64_t& smem) {
    if (n2 % 4 != 0 || n2 < 8 || n2 > 2048) return false;
    g.BK = n2;  // whole rows: every copy is a 1-D bulk copy of consecutive rows
    const int per128 = 128 / es;
    g.pitch = (n2 + per128 - 1) / per128 * per128;
    const int tpr = n2 / 4;
    g.tab_bytes = round128((int)smem_table);
    g.CI = g_force_ci > 0 ? g_force_ci : 64;
    if (g.CI > nplanes) g.CI = nplanes;
    g.bal = 0;
    // Candidates: TJ with TJ*tpr consumers a multiple of 32 in [32, 512], ring
    // depth S in [3, 5].  Score = consumer warps per SM x TJ/(TJ+2) (the share
    // of loaded rows that are not halo), deeper rings preferred on ties.
    double best = -1.0;
    MarchGeom pick{};
    for (int tj = 1; tj <= 64; ++tj) {
        if (g_force_tj > 0 && tj != g_force_tj) continue;
        if (n1 % tj || (tj * tpr) % 32 || tj * tpr > 512) continue;
        for (int st = 3; st <= 5; ++st) {
            if (g_force_stages > 0 && st != g_force_stages) continue;
            MarchGeom c = g;
            c.TJ = tj;
            c.S = st;
            c.stage_bytes = comps * round128((tj + 2) * c.pitch * es);
            if (smem_need(c) > kSmemPerCta) continue;
            const int cps = ctas_per_sm(c, tpr);
            if (cps < 1) continue;
            const double score = cps * (tj * tpr / 32) * (double)tj / (tj + 2) + 0.01 * st;
            if (score > best) {
                best = score;
                pick = c;
            }
        }
    }
    if (best < 0) return false;
    g = pick;
    // bulk-copy destinations (ring + stage*stage_bytes + block*stage_bytes/blocks +
    // rr*pitch*es) are 128-byte aligned; sources and sizes are multiples of the
    // 16-byte row length (n2 % 4 == 0)
    if ((g.pitch * es) % 128 || g.stage_bytes % (128 * comps) || g.tab_bytes % 128) return false;
    g.nJB = n1 / g.TJ;
    g.nIC = (nplanes + g.CI - 1) / g.CI;
    g.items = g.nJB * g.nIC;
    smem = smem_need(g);
    return true;
}

static bool geometry(int storage, const RealStageParams& p, int64_t smem_table, MarchGeom& g,
                     int64_t& smem) {
    return geometry_dims(p.n1, p.n2, p.i_end - p.i_begin, layout_es(storage),
                         2 * layout_planes(storage), smem_table, g, smem);
}

bool march_supported(int storage, const RealStageParams& p) {
    if (storage != TIPT_F32C && storage != TIPT_F64 && storage != TIPT_F32) return false;
    if (storage != TIPT_F32C && p.range) return false;  // the generic kernel folds the range
    const uintptr_t a = reinterpret_cast<uintptr_t>(p.phi) | reinterpret_cast<uintptr_t>(p.pi) |
                        reinterpret_cast<uintptr_t>(p.phi_out) |
                        reinterpret_cast<uintptr_t>(p.pi_out);
    if (a % 16) return false;
    MarchGeom g;
    int64_t smem;
    int64_t tb = p.table_in_smem ? (int64_t)p.npts * (storage == TIPT_F32C ? 4 : 8) : 0;
    return geometry(storage, p, tb, g, smem);
}

template <typename Kern, typename... Extra>
static int launch_march_k(Kern kern, const RealStageParams& p, const MarchGeom& g, int64_t smem,
                          cudaStream_t st, Extra... extra) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return fail_cuda(e, "marching kernel attributes");
    const int threads = g.TJ * (p.n2 / 4) + 32;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, (size_t)smem);
    if (e != cudaSuccess || per_sm < 1)
        return fail(TIPT_ERR_UNSUPPORTED, "marching kernel does not fit an SM (%d threads, %lld "
                    "bytes of shared memory)", threads, (long long)smem);
    int grid = num_sms() * per_sm;
    if (grid > g.items) grid = g.items;
    kern<<<grid, threads, (size_t)smem, st>>>(p, g, extra...);
    e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "marching kernel launch");
}

// The batched ensemble's replicas of one 3-D shape class (n0, n1, n2 with
// n2 % 4 == 0) on the compensated-FP32 marching stage: rids[0..n_rids) are the
// class's replica ids; p carries the shared step constants (dt, dx, eta, mu,
// inv_a2), the packed state pointers and the class shape.
int launch_ensemble_march(const RealStageParams& p_in, const tipt_replica* reps,
                          const int32_t* rids, int n_rids, const int32_t* n_rids_dev,
                          const int32_t* active, int64_t n_total,
                          const unsigned long long* ctr, long long offset, cudaStream_t st) {
    RealStageParams p = p_in;
    p.i_begin = 0;
    p.i_end = p.n0;
    p.vkind = TIPT_VP_POLY;
    p.table_in_smem = 0;
    p.mul = kPass2Mul;
    set_f32c_pairs(p);
    MarchGeom g;
    int64_t smem;
    if (!geometry(TIPT_F32C, p, 0, g, smem))
        return fail(TIPT_ERR_UNSUPPORTED, "no marching geometry for the replica shape");
    // 32-plane chunks: work items small enough to spread a few active replicas
    // over the SMs
    if (g_force_ci == 0 && g.CI > 32) {
        g.CI = 32;
        g.nIC = (p.n0 + g.CI - 1) / g.CI;
        g.items = g.nJB * g.nIC;
    }
    g.bal = 0;  // replica work items only
    EnsMarch em;
    em.reps = reps;
    em.rids = rids;
    em.n_rids = n_rids_dev;
    em.active = active;
    em.n_total = n_total;
    em.items_per_rep = g.items;
    em.step = p.step;
    em.ctr = ctr;
    em.offset = offset;
    if ((int64_t)g.items * n_rids > 0x7FFFFFFF)
        return fail(TIPT_ERR_UNSUPPORTED, "too many work items");
    g.items *= n_rids;
    // 64-bit noise-key sites when a replica's site index can exceed 32 bits
    const bool wide = (int64_t)p.n0 * p.n1 * p.n2 > 0xFFFFFFFFll;
    // the classes of the batched configuration (64^3: 32-row tiles, 96^3: 16-row
    // tiles) run kernels compiled for their geometry
    const bool exact = g_fixed_geom && !wide && g.pitch == p.n2 &&
                       g.stage_bytes == 4 * (g.TJ + 2) * g.pitch * 4;
    if (exact && p.n2 == 64 && g.TJ == 32)
        return launch_march_k(rk2_stage_march_f32c<false, false, false, true, 64, 32>, p, g, smem, st,
                              em);
    if (exact && p.n2 == 96 && g.TJ == 16)
        return launch_march_k(rk2_stage_march_f32c<false, false, false, true, 96, 16>, p, g, smem, st,
                              em);
    return wide ? launch_march_k(rk2_stage_march_f32c<true, false, false, true>, p, g, smem, st, em)
                : launch_march_k(rk2_stage_march_f32c<false, false, false, true>, p, g, smem, st, em);
}

bool ensemble_march_supported(int n0, int n1, int n2) {
    if (n0 < 2 || n2 % 4 != 0) return false;
    RealStageParams p;
    memset(&p, 0, sizeof(p));
    p.n0 = n0;
    p.n1 = n1;
    p.n2 = n2;
    p.i_begin = 0;
    p.i_end = n0;
    MarchGeom g;
    int64_t smem;
    return geometry(TIPT_F32C, p, 0, g, smem);
}

// Compensated-FP32 stage with a table or polynomial V'.  With the V' row staged
// in shared memory and hash noise (TAB): the kernel compiled for 512-site rows
// in 4-row tiles or 256-site rows in 8-row tiles when the run-time geometry is
// exactly that one (the automatic choice at 512^3 and 256^3), else the
// run-time-geometry TAB kernel; otherwise the dispatching kernel.  All give the
// same bits.
template <bool WIDE, bool RG>
static int launch_f32c_stage(const RealStageParams& q, const MarchGeom& g0, int64_t smem0,
                             int64_t smem_table, cudaStream_t st) {
    const bool tab = q.table_in_smem && (q.vkind == TIPT_VP_TABLE || q.vkind == TIPT_VP_TABLE2D) &&
                     !q.noise;
    // lattices with fewer CI-plane items than SMs: every CTA an equal share of the
    // (j-block, plane) units, so every SM works.  (With more items the round-robin
    // items stay: they keep the CTAs of neighbouring j-blocks at the same planes,
    // so a tile's halo rows are still in L2 from the neighbour's reads; the
    // j-block-major shares lose that reuse and measured 6 % slower at 512^3.)
    const auto balance = [&](MarchGeom& b) {
        if (!g_balance || b.items >= num_sms()) return;
        b.bal = 1;
        const int64_t units = (int64_t)b.nJB * (q.i_end - q.i_begin);
        b.items = units < 0x7FFFFFFF ? (int)units : 0x7FFFFFFF;
    };
    // the TAB kernels stage the row as (value, slope) pairs: twice the table bytes
    MarchGeom g;
    int64_t smem;
    if (!tab || !geometry(TIPT_F32C, q, 2 * smem_table, g, smem)) {
        MarchGeom b = g0;
        balance(b);
        return launch_march_k(rk2_stage_march_f32c<WIDE, false, RG, false>, q, b, smem0, st,
                              EnsMarch{});
    }
    balance(g);
    const bool exact = g_fixed_geom && g.pitch == q.n2 &&
                       g.stage_bytes == 4 * (g.TJ + 2) * g.pitch * 4;
    if (exact && q.n2 == 512 && g.TJ == 4)
        return launch_march_k(rk2_stage_march_f32c<WIDE, false, RG, false, 512, 4, true>, q, g,
                              smem, st, EnsMarch{});
    if (exact && q.n2 == 256 && g.TJ == 8)
        return launch_march_k(rk2_stage_march_f32c<WIDE, false, RG, false, 256, 8, true>, q, g,
                              smem, st, EnsMarch{});
    return launch_march_k(rk2_stage_march_f32c<WIDE, false, RG, false, 0, 0, true>, q, g, smem, st,
                          EnsMarch{});
}

int launch_march(int storage, const RealStageParams& p, int64_t smem_table, cudaStream_t st) {
    MarchGeom g;
    int64_t smem;
    if (!geometry(storage, p, smem_table, g, smem))
        return fail(TIPT_ERR_UNSUPPORTED, "marching kernel geometry");
    // 64-bit noise-key sites when an index (array + offset) can exceed 32 bits
    const bool wide = (int64_t)p.n0 * p.n1 * p.n2 + (p.site_offset > 0 ? p.site_offset : 0) >
                      0xFFFFFFFFll;
    if (storage == TIPT_F32C && p.vkind == TIPT_VP_THERMAL) {
        if (p.range)
            return wide ? launch_march_k(rk2_stage_march_f32c<true, true, true, false>, p, g, smem, st, EnsMarch{})
                        : launch_march_k(rk2_stage_march_f32c<false, true, true, false>, p, g, smem, st, EnsMarch{});
        return wide ? launch_march_k(rk2_stage_march_f32c<true, true, false, false>, p, g, smem, st, EnsMarch{})
                    : launch_march_k(rk2_stage_march_f32c<false, true, false, false>, p, g, smem, st, EnsMarch{});
    }
    if (storage == TIPT_F32C) {
        RealStageParams q = p;
        q.test_withhold = g_test_withhold;
        g_test_withhold = 0;
        if (q.range)
            return wide ? launch_f32c_stage<true, true>(q, g, smem, smem_table, st)
                        : launch_f32c_stage<false, true>(q, g, smem, smem_table, st);
        return wide ? launch_f32c_stage<true, false>(q, g, smem, smem_table, st)
                    : launch_f32c_stage<false, false>(q, g, smem, smem_table, st);
    }
    if (storage != TIPT_F32C && p.range)
        return fail(TIPT_ERR_UNSUPPORTED, "the FP64 / float32 marching stage takes no range output");
    if (storage == TIPT_F64)
        return wide ? launch_march_k(rk2_stage_march<TIPT_F64, true>, p, g, smem, st)
                    : launch_march_k(rk2_stage_march<TIPT_F64, false>, p, g, smem, st);
    if (storage == TIPT_F32)
        return wide ? launch_march_k(rk2_stage_march<TIPT_F32, true>, p, g, smem, st)
                    : launch_march_k(rk2_stage_march<TIPT_F32, false>, p, g, smem, st);
    return fail(TIPT_ERR_STORAGE, "marching kernel takes F32C, F64 or F32");
}

// The alternative integrators on the marching ring: compensated FP32,
// polynomial V' or a table staged in shared memory, n2 % 4 == 0; the complex
// field without Z_N (its force runs in FP64 on the generic kernel).
static bool alt_geometry(const AltParams& p, bool cplx, MarchGeom& g, int64_t& smem) {
    if (p.v.vkind != TIPT_VP_POLY && !p.v.table_in_smem) return false;
    if (cplx && p.v.zn_active > 0.5 && p.v.zn_n > 0.5) return false;
    const int64_t tb = p.v.vkind == TIPT_VP_POLY ? 0 : (int64_t)p.v.npts * 4;
    return geometry_dims(p.n1, p.n2, p.n0, 4, cplx ? 4 : 2, tb, g, smem);
}

bool alt_march_supported(const AltParams& p, bool cplx) {
    uintptr_t a = 0;
    for (int q = 0; q < (cplx ? 4 : 2); ++q)
        a |= reinterpret_cast<uintptr_t>(p.f[q]) | reinterpret_cast<uintptr_t>(p.o[q]);
    if (a % 16) return false;
    MarchGeom g;
    int64_t smem;
    return alt_geometry(p, cplx, g, smem);
}

template <int MODE, bool CPLX>
static int launch_alt_march_k(const AltParams& p, cudaStream_t st) {
    MarchGeom g;
    int64_t smem;
    if (!alt_geometry(p, CPLX, g, smem))
        return fail(TIPT_ERR_UNSUPPORTED, "integrator march geometry");
    const bool wide = (int64_t)p.n0 * p.n1 * p.n2 > 0xFFFFFFFFll;
    // the staged table fixed at compile time where the run uses it (the complex
    // force with or without the eps term)
    const bool tab = p.v.vkind != TIPT_VP_POLY && p.v.table_in_smem;
    const int src = !tab ? kCsrcAny : (CPLX && p.v.eps4 != 0.0) ? kCsrcTabEps : kCsrcTab;
    // rows of 512 sites in 4-row tiles (the automatic choice at 512^3) with the
    // staged table: the geometry fixed at compile time as well
    constexpr int NF = CPLX ? 2 : 1;
    const bool fixed = g_fixed_geom && tab && p.n2 == 512 && g.pitch == 512 && g.TJ == 4 &&
                       g.stage_bytes == 2 * NF * 6 * 512 * 4;
    constexpr int TS = CPLX ? kCsrcTabEps : kCsrcTab;
    auto kern = fixed ? (src == kCsrcTab
                             ? (wide ? alt_march_f32c<MODE, CPLX, true, kCsrcTab, 512, 4>
                                     : alt_march_f32c<MODE, CPLX, false, kCsrcTab, 512, 4>)
                             : (wide ? alt_march_f32c<MODE, CPLX, true, TS, 512, 4>
                                     : alt_march_f32c<MODE, CPLX, false, TS, 512, 4>))
                : src == kCsrcTab
                    ? (wide ? alt_march_f32c<MODE, CPLX, true, kCsrcTab>
                            : alt_march_f32c<MODE, CPLX, false, kCsrcTab>)
                : src == kCsrcTabEps
                    ? (wide ? alt_march_f32c<MODE, CPLX, true, CPLX ? kCsrcTabEps : kCsrcTab>
                            : alt_march_f32c<MODE, CPLX, false, CPLX ? kCsrcTabEps : kCsrcTab>)
                    : (wide ? alt_march_f32c<MODE, CPLX, true> : alt_march_f32c<MODE, CPLX, false>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return fail_cuda(e, "integrator march attributes");
    const int threads = g.TJ * (p.n2 / 4) + 32;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, (size_t)smem);
    if (e != cudaSuccess || per_sm < 1)
        return fail(TIPT_ERR_UNSUPPORTED, "integrator march kernel does not fit an SM");
    int grid = num_sms() * per_sm;
    if (grid > g.items) grid = g.items;
    kern<<<grid, threads, (size_t)smem, st>>>(p, g);
    e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "integrator march launch");
}

int launch_alt_march(int mode, bool cplx, const AltParams& p, cudaStream_t st) {
    if (cplx) {
        switch (mode) {
            case kOD: return launch_alt_march_k<kOD, true>(p, st);
            case kBA1: return launch_alt_march_k<kBA1, true>(p, st);
            default: return launch_alt_march_k<kBA2, true>(p, st);
        }
    }
    switch (mode) {
        case kOD: return launch_alt_march_k<kOD, false>(p, st);
        case kBA1: return launch_alt_march_k<kBA1, false>(p, st);
        default: return launch_alt_march_k<kBA2, false>(p, st);
    }
}

// Complex F32C geometry: two sites per consumer thread (tpr = n2/2 per row),
// eight planes per ring stage; the same scoring as the real field.
static int g_force_kseg = 0;  // complex kernel's row segment (0 = automatic)

// Candidates: segments KS dividing n2 (split segments of at least 128 sites and a
// multiple of 32), TJ with TJ*KS/2 consumers a multiple of 32 in
// [32, 512], ring depth S in [3, 5].  Score: consumer warps per SM x TJ/(TJ+2),
// weighted by ring depth (a 3-stage ring prefetches nothing beyond the plane in
// use) and by segment length.
static bool complex_geometry(const ComplexStageParams& p, MarchGeom& g, int64_t& smem) {
    const int n1 = p.n1, n2 = p.n2;
    const int es = 4, np = 8;
    if (n2 % 2 != 0 || n2 < 16 || n2 > 1024) return false;
    g.tab_bytes = p.table_in_smem ? round128(p.npts * 4) : 0;
    g.CI = g_force_ci > 0 ? g_force_ci : 64;
    if (g.CI > p.n0) g.CI = p.n0;
    double best = -1.0;
    MarchGeom pick{};
    for (int ks = n2; ks >= 16; --ks) {
        if (n2 % ks) continue;
        const bool split = ks != n2;
        if (g_force_kseg > 0 && ks != g_force_kseg) continue;
        if (split && (ks % 32 || ks < 128)) continue;
        MarchGeom b = g;
        b.KS = ks;
        b.nKS = n2 / ks;
        b.BK = pick_bk(ks, es);
        if (!b.BK) continue;
        b.pitch = (ks + 31) / 32 * 32;
        const int tpr = ks / 2;
        for (int tj = 1; tj <= 64; ++tj) {
            if (g_force_tj > 0 && tj != g_force_tj) continue;
            if (n1 % tj || (tj * tpr) % 32 || tj * tpr > 512) continue;
            for (int st = 3; st <= 5; ++st) {
                if (g_force_stages > 0 && st != g_force_stages) continue;
                MarchGeom c = b;
                c.TJ = tj;
                c.S = st;
                c.halo_off = np * round128((tj + 2) * c.pitch * es);
                c.stage_bytes = c.halo_off;
                if (smem_need(c) + (split ? tj * 2 * 16 * 4 : 0) > kSmemPerCta) continue;
                const int cps = ctas_per_sm(c, tpr);
                if (cps < 1) continue;
                // measured at 512^3 and 256^3: ring depth and long segments (fewer,
                // larger copies) outweigh consumer warps
                const double depth = st >= 5 ? 1.0 : (st == 4 ? 0.85 : 0.3);
                const double seg = ks >= 256 || !split ? 1.0 : ks / 256.0;
                const double score = cps * (tj * tpr / 32) * (double)tj / (tj + 2) * depth * seg +
                                     0.001 * ks / n2;
                if (score > best) {
                    best = score;
                    pick = c;
                }
            }
        }
    }
    if (best < 0) return false;
    g = pick;
    if ((g.pitch * es) % 128 || ((g.BK * es) % 128 && g.BK != g.KS) || (g.BK * es) % 16 ||
        g.halo_off % (128 * np) || g.tab_bytes % 128)
        return false;
    g.nJB = n1 / g.TJ;
    g.nIC = (p.n0 + g.CI - 1) / g.CI;
    g.items = g.nJB * g.nKS * g.nIC;
    smem = smem_need(g) + (g.nKS > 1 ? g.TJ * 2 * 16 * 4 : 0);
    return true;
}

bool complex_march_supported(const ComplexStageParams& p) {
    if (p.noise1 || (p.zn_active > 0.5 && p.zn_n > 0.5)) return false;
    if (p.vkind != TIPT_VP_POLY && !p.table_in_smem) return false;
    if (!encode_fn()) return false;
    uintptr_t a = 0;
    for (int f = 0; f < 4; ++f)
        a |= reinterpret_cast<uintptr_t>(p.f[f]) | reinterpret_cast<uintptr_t>(p.o[f]);
    if (a % 16) return false;
    MarchGeom g;
    int64_t smem;
    return complex_geometry(p, g, smem);
}

int launch_complex_march(const ComplexStageParams& p, cudaStream_t st) {
    MarchGeom g;
    int64_t smem;
    if (!complex_geometry(p, g, smem))
        return fail(TIPT_ERR_UNSUPPORTED, "complex marching kernel geometry");
    const bool wide = (int64_t)p.n0 * p.n1 * p.n2 > 0xFFFFFFFFll;
    CUtensorMap tm[4];
    for (int f = 0; f < 4; ++f)
        if (!make_map(&tm[f], p.f[f], 2 * p.n0, p.n1, p.n2, 4, g.BK))
            return fail(TIPT_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    // 256-site segments in 4-row tiles (the automatic choice at 256^3 and 512^3)
    // compiled with that geometry fixed
    const bool fixed = g_fixed_geom && g.KS == 256 && g.TJ == 4 && g.pitch == 256 &&
                       g.halo_off == 8 * 6 * 256 * 4 && g.stage_bytes == g.halo_off;
    auto kern = fixed ? (p.range ? (wide ? complex_stage_march_f32c<true, true, 256, 4>
                                         : complex_stage_march_f32c<false, true, 256, 4>)
                                 : (wide ? complex_stage_march_f32c<true, false, 256, 4>
                                         : complex_stage_march_f32c<false, false, 256, 4>))
            : p.range ? (wide ? complex_stage_march_f32c<true, true> : complex_stage_march_f32c<false, true>)
                      : (wide ? complex_stage_march_f32c<true, false> : complex_stage_march_f32c<false, false>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return fail_cuda(e, "complex marching kernel attributes");
    const int threads = g.TJ * (g.KS / 2) + 32;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, (size_t)smem);
    if (e != cudaSuccess || per_sm < 1)
        return fail(TIPT_ERR_UNSUPPORTED, "complex marching kernel does not fit an SM (%d "
                    "threads, %lld bytes of shared memory)", threads, (long long)smem);
    int grid = num_sms() * per_sm;
    if (grid > g.items) grid = g.items;
    kern<<<grid, threads, (size_t)smem, st>>>(tm[0], tm[1], tm[2], tm[3], p, g);
    e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "complex marching kernel launch");
}

}  // namespace tipt

using namespace tipt;

// Tile shape of the marching kernel: rows per tile, planes per i-chunk and
// ring stages (0 = automatic).  Used by the autotuner; performance only.
// Row segment of the complex marching kernel (0 = automatic); performance only.
extern "C" int tipt_set_march_kseg(int kseg) {
    if (kseg < 0) return fail(TIPT_ERR_ARG, "bad row segment");
    g_force_kseg = kseg;
    return TIPT_OK;
}

// The compensated-FP32 marching kernels compiled for fixed geometries (real and
// complex stages, integrators, ensemble classes) on or off; performance only
// (they give the run-time-geometry kernels' bits).
extern "C" int tipt_set_march_fixed(int enable) {
    g_fixed_geom = enable != 0;
    return TIPT_OK;
}

extern "C" int tipt_set_march_tiles(int rows, int planes, int stages) {
    if (rows < 0 || planes < 0 || stages < 0 || (stages > 0 && stages < 3) || stages > 5)
        return fail(TIPT_ERR_ARG, "bad tile shape");
    g_force_tj = rows;
    g_force_ci = planes;
    g_force_stages = stages;
    return TIPT_OK;
}

// Test of the bounded device waits: the next compensated-FP32 marching stage
// launch (polynomial or table V') withholds ring position `position` (>= 0) in
// its block 0 -- no copy is issued for it or after it, so nothing is left in
// flight -- and the consumers of that block give up waiting after the bounded
// wait (2 s), record TIPT_ERR_TIMEOUT and return.  position < 0 disarms.
extern "C" int tipt_test_withhold_plane(int position) {
    g_test_withhold = position >= 0 ? position + 1 : 0;
    return TIPT_OK;
}

// Reads (and with clear != 0 resets) the device status word that bounded
// device-side waits set on expiry.  Synchronises the device.
extern "C" int tipt_device_status(int* status, int clear) {
    if (!status) return fail(TIPT_ERR_ARG, "status is NULL");
    cudaError_t e = cudaMemcpyFromSymbol(status, g_device_status, sizeof(int));
    if (e != cudaSuccess) return fail_cuda(e, "read device status");
    if (clear) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_device_status, &zero, sizeof(int));
        if (e != cudaSuccess) return fail_cuda(e, "clear device status");
    }
    int other = 0;
    int rc = mlp_status(&other, clear);
    if (rc) return rc;
    if (!*status) *status = other;
    other = 0;
    if ((rc = label_status(&other, clear))) return rc;
    if (!*status) *status = other;
    return TIPT_OK;
}
