// Connected-component labelling of thresholded lattice fields: bubbles
// (|phi| > threshold) and string voxels (|winding| > 0.5), the GPU
// replacement of scipy.ndimage.label in the reference's post-processing
// (postprocess/revisualize_snapshots.py:171-214 _identify_bubbles, :360-392
// _identify_strings).
//
// Connectivity is the face-neighbour (6-connected) structure of
// scipy.ndimage.label's default; the lattice is open (non-periodic) like
// scipy's, or periodic on request.  Labels are numbered 1..n in raster order
// of each component's first voxel, which is scipy's numbering, so the label
// array is identical.
//
// Method (union-find with atomic-min hooking, Playne & Hawick, "A new
// algorithm for parallel connected-component labelling on GPUs", IEEE TPDS
// 2018): every masked site starts as its own root; each site unites with its
// +x, +y, +z masked neighbours by hooking the larger root under the smaller
// one with atomicMin, so a component's root ends as its smallest linear
// index; a pass of path compression leaves every site pointing at its root;
// roots are ranked in index order (per-chunk counts, one scan, per-chunk
// ballots) and the ranks are gathered back to the sites.  Every chase loop is
// bounded; an exhausted bound sets the status word to TIPT_ERR_TIMEOUT.
#include "tipt_device.cuh"
#include "tipt_internal.h"

namespace tipt {

constexpr int kChunk = 8192;        // sites per ranking chunk
constexpr int kChase = 1 << 24;     // bound on any find / unite loop

__device__ int g_label_status = 0;

template <int S>
__device__ __forceinline__ double field_abs(const void* f, int64_t s, int64_t N) {
    if constexpr (S == TIPT_F64) return fabs(__ldg(static_cast<const double*>(f) + s));
    else if constexpr (S == TIPT_F32) return fabs((double)__ldg(static_cast<const float*>(f) + s));
    else {
        const float* p = static_cast<const float*>(f);
        return fabs((double)__ldg(p + s) + (double)__ldg(p + N + s));
    }
}
template <int S>
__device__ __forceinline__ double field_val(const void* f, int64_t s, int64_t N) {
    if constexpr (S == TIPT_F64) return __ldg(static_cast<const double*>(f) + s);
    else if constexpr (S == TIPT_F32) return (double)__ldg(static_cast<const float*>(f) + s);
    else {
        const float* p = static_cast<const float*>(f);
        return (double)__ldg(p + s) + (double)__ldg(p + N + s);
    }
}

template <int S>
__global__ void label_init_kernel(const void* f, double thr, int32_t* L, int64_t N) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x)
        L[s] = field_abs<S>(f, s, N) > thr ? (int32_t)s : -1;
}

__device__ __forceinline__ int32_t find_root(const int32_t* L, int32_t x, bool& ok) {
    for (int it = 0; it < kChase; ++it) {
        const int32_t y = L[x];
        if (y == x) return x;
        x = y;
    }
    ok = false;
    return x;
}

__device__ __forceinline__ void unite(int32_t* L, int32_t a, int32_t b, bool& ok) {
    for (int it = 0; it < kChase && ok; ++it) {
        a = find_root(L, a, ok);
        b = find_root(L, b, ok);
        if (a == b) return;
        if (a < b) {
            const int32_t old = atomicMin(&L[b], a);
            if (old == b) return;
            b = old;
        } else {
            const int32_t old = atomicMin(&L[a], b);
            if (old == a) return;
            a = old;
        }
    }
    ok = false;
}

__global__ void label_merge_kernel(int32_t* L, int n0, int n1, int n2, int periodic) {
    const int64_t n12 = (int64_t)n1 * n2, N = (int64_t)n0 * n12;
    bool ok = true;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        if (L[s] < 0) continue;
        const int k = (int)(s % n2);
        const int64_t r = s / n2;
        const int j = (int)(r % n1);
        const int i = (int)(r / n1);
        int64_t nb[3] = {-1, -1, -1};
        if (i + 1 < n0) nb[0] = s + n12;
        else if (periodic && n0 > 1) nb[0] = s - (int64_t)(n0 - 1) * n12;
        if (j + 1 < n1) nb[1] = s + n2;
        else if (periodic && n1 > 1) nb[1] = s - (int64_t)(n1 - 1) * n2;
        if (k + 1 < n2) nb[2] = s + 1;
        else if (periodic && n2 > 1) nb[2] = s - (n2 - 1);
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (nb[d] >= 0 && L[nb[d]] >= 0) unite(L, (int32_t)s, (int32_t)nb[d], ok);
    }
    if (!ok) atomicExch(&g_label_status, (int)TIPT_ERR_TIMEOUT);
}

__global__ void label_compress_kernel(int32_t* L, int64_t N) {
    bool ok = true;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x)
        if (L[s] >= 0) L[s] = find_root(L, L[s], ok);
    if (!ok) atomicExch(&g_label_status, (int)TIPT_ERR_TIMEOUT);
}

// roots per chunk (a root is a masked site that is its own label)
__global__ void label_count_kernel(const int32_t* L, int64_t N, int32_t* chunk_roots) {
    __shared__ int32_t s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    const int64_t b0 = (int64_t)blockIdx.x * kChunk;
    int32_t c = 0;
    for (int64_t s = b0 + threadIdx.x; s < b0 + kChunk && s < N; s += blockDim.x) c += L[s] == (int32_t)s;
    atomicAdd(&s_cnt, c);
    __syncthreads();
    if (threadIdx.x == 0) chunk_roots[blockIdx.x] = s_cnt;
}

// exclusive scan of the chunk counts (one block) and the total
__global__ void label_scan_kernel(int32_t* chunk_roots, int n_chunks, int32_t* n_labels) {
    __shared__ int32_t s_part[1024];
    const int per = (n_chunks + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per;
    int32_t sum = 0;
    for (int q = b; q < b + per && q < n_chunks; ++q) sum += chunk_roots[q];
    s_part[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t run = 0;
        for (int t = 0; t < (int)blockDim.x; ++t) {
            const int32_t v = s_part[t];
            s_part[t] = run;
            run += v;
        }
        *n_labels = run;
    }
    __syncthreads();
    int32_t run = s_part[threadIdx.x];
    for (int q = b; q < b + per && q < n_chunks; ++q) {
        const int32_t v = chunk_roots[q];
        chunk_roots[q] = run;
        run += v;
    }
}

// rank the roots of a chunk in index order: R[root] = label (1-based)
__global__ void label_rank_kernel(const int32_t* L, int64_t N, const int32_t* chunk_base,
                                  int32_t* R) {
    __shared__ int32_t s_warp[33];
    const int64_t b0 = (int64_t)blockIdx.x * kChunk;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int32_t base = chunk_base[blockIdx.x];
    for (int64_t off = 0; off < kChunk; off += blockDim.x) {
        const int64_t s = b0 + off + threadIdx.x;
        const bool root = s < N && L[s] == (int32_t)s;
        const unsigned m = __ballot_sync(0xffffffffu, root);
        if (lane == 0) s_warp[warp] = __popc(m);
        __syncthreads();
        if (threadIdx.x == 0) {
            int32_t run = 0;
            for (int w = 0; w < nw; ++w) {
                const int32_t v = s_warp[w];
                s_warp[w] = run;
                run += v;
            }
            s_warp[32] = run;
        }
        __syncthreads();
        if (root) R[s] = base + s_warp[warp] + __popc(m & ((1u << lane) - 1u)) + 1;
        base += s_warp[32];
        __syncthreads();
    }
}

__global__ void label_gather_kernel(const int32_t* L, const int32_t* R, int32_t* out, int64_t N) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l = L[s];
        out[s] = l < 0 ? 0 : R[l];
    }
}

// per-label statistics (index 0 = background, left at zero)
struct LabelStats {
    int64_t* count;     // [n+1]
    int64_t* sum_xyz;   // [n+1][3]
    int64_t* sum_sq;    // [n+1]  sum of x^2 + y^2 + z^2
    double* sum_val;    // [n+1]
    double* max_abs;    // [n+1]
};

__global__ void stats_zero_kernel(LabelStats st, int64_t n1) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n1;
         q += (int64_t)gridDim.x * blockDim.x) {
        st.count[q] = 0;
        st.sum_xyz[3 * q] = st.sum_xyz[3 * q + 1] = st.sum_xyz[3 * q + 2] = 0;
        st.sum_sq[q] = 0;
        st.sum_val[q] = 0.0;
        st.max_abs[q] = 0.0;
    }
}

template <int S>
__global__ void stats_kernel(const void* f, const int32_t* lab, int n0, int n1, int n2,
                             int32_t n_labels, LabelStats st) {
    const int64_t n12 = (int64_t)n1 * n2, N = (int64_t)n0 * n12;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l = lab[s];
        if (l <= 0 || l > n_labels) continue;
        const int64_t k = s % n2, r = s / n2, j = r % n1, i = r / n1;
        const double v = f ? field_val<S>(f, s, N) : 0.0;
        atomicAdd(reinterpret_cast<unsigned long long*>(&st.count[l]), 1ull);
        atomicAdd(reinterpret_cast<unsigned long long*>(&st.sum_xyz[3 * l]), (unsigned long long)i);
        atomicAdd(reinterpret_cast<unsigned long long*>(&st.sum_xyz[3 * l + 1]), (unsigned long long)j);
        atomicAdd(reinterpret_cast<unsigned long long*>(&st.sum_xyz[3 * l + 2]), (unsigned long long)k);
        atomicAdd(reinterpret_cast<unsigned long long*>(&st.sum_sq[l]),
                  (unsigned long long)(i * i + j * j + k * k));
        atomicAdd(&st.sum_val[l], v);
        // |v| >= 0: the IEEE bit patterns of non-negative doubles order like the values
        atomicMax(reinterpret_cast<unsigned long long*>(&st.max_abs[l]),
                  (unsigned long long)__double_as_longlong(fabs(v)));
    }
}

static int grid_for(int64_t N) {
    int64_t b = (N + 255) / 256;
    const int64_t cap = (int64_t)num_sms() * 16;
    return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

int64_t label_workspace_bytes(int64_t N) {
    const int64_t chunks = (N + kChunk - 1) / kChunk;
    return 4 * (2 * N + chunks + 64);
}

// Read (and optionally clear) the labeller's status word.
int label_status(int* status, int clear) {
    cudaError_t e = cudaMemcpyFromSymbol(status, g_label_status, sizeof(int));
    if (e == cudaSuccess && clear) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_label_status, &zero, sizeof(int));
    }
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "label status");
}

}  // namespace tipt

using namespace tipt;

extern "C" int64_t tipt_label_workspace_size(int64_t nx, int64_t ny, int64_t nz) {
    if (nx < 1 || ny < 1 || nz < 1) return 0;
    return label_workspace_bytes(nx * ny * nz);
}

extern "C" int tipt_label_components(int storage, const void* field, double threshold,
                                     int64_t nx, int64_t ny, int64_t nz, int periodic,
                                     int32_t* labels, int32_t* n_labels, void* workspace,
                                     int64_t workspace_bytes, void* stream) {
    int rc;
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz))) return rc;
    const int64_t N = nx * ny * nz;
    if (N >= (1ll << 31)) return fail(TIPT_ERR_UNSUPPORTED, "labelling takes < 2^31 sites");
    if ((rc = check_ptr(field, elem_align(storage), "field")) ||
        (rc = check_ptr(labels, 4, "labels")) || (rc = check_ptr(n_labels, 4, "n_labels")) ||
        (rc = check_ptr(workspace, 4, "workspace")))
        return rc;
    if (workspace_bytes < label_workspace_bytes(N))
        return fail(TIPT_ERR_ARG, "workspace of %lld bytes is smaller than the %lld needed",
                    (long long)workspace_bytes, (long long)label_workspace_bytes(N));
    const int64_t chunks = (N + kChunk - 1) / kChunk;
    int32_t* L = static_cast<int32_t*>(workspace);
    int32_t* R = L + N;
    int32_t* cr = R + N;
    cudaStream_t st = (cudaStream_t)stream;
    const int g = grid_for(N);
    switch (storage) {
        case TIPT_F64: label_init_kernel<TIPT_F64><<<g, 256, 0, st>>>(field, threshold, L, N); break;
        case TIPT_F32: label_init_kernel<TIPT_F32><<<g, 256, 0, st>>>(field, threshold, L, N); break;
        default: label_init_kernel<TIPT_F32C><<<g, 256, 0, st>>>(field, threshold, L, N); break;
    }
    label_merge_kernel<<<g, 256, 0, st>>>(L, (int)nx, (int)ny, (int)nz, periodic ? 1 : 0);
    label_compress_kernel<<<g, 256, 0, st>>>(L, N);
    label_count_kernel<<<(unsigned)chunks, 256, 0, st>>>(L, N, cr);
    label_scan_kernel<<<1, 1024, 0, st>>>(cr, (int)chunks, n_labels);
    label_rank_kernel<<<(unsigned)chunks, 256, 0, st>>>(L, N, cr, R);
    label_gather_kernel<<<g, 256, 0, st>>>(L, R, labels, N);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "labelling launch");
}

extern "C" int tipt_label_stats(int storage, const void* field, const int32_t* labels, int64_t nx,
                                int64_t ny, int64_t nz, int32_t n_labels, int64_t* count,
                                int64_t* sum_xyz, int64_t* sum_sq, double* sum_val,
                                double* max_abs, void* stream) {
    int rc;
    if ((rc = check_storage(storage)) || (rc = check_dims(nx, ny, nz))) return rc;
    if (field && (rc = check_ptr(field, elem_align(storage), "field"))) return rc;
    if ((rc = check_ptr(labels, 4, "labels")) || (rc = check_ptr(count, 8, "count")) ||
        (rc = check_ptr(sum_xyz, 8, "sum_xyz")) || (rc = check_ptr(sum_sq, 8, "sum_sq")) ||
        (rc = check_ptr(sum_val, 8, "sum_val")) || (rc = check_ptr(max_abs, 8, "max_abs")))
        return rc;
    if (n_labels < 0) return fail(TIPT_ERR_ARG, "n_labels < 0");
    const int64_t N = nx * ny * nz;
    LabelStats s{count, sum_xyz, sum_sq, sum_val, max_abs};
    cudaStream_t st = (cudaStream_t)stream;
    stats_zero_kernel<<<grid_for(n_labels + 1), 256, 0, st>>>(s, (int64_t)n_labels + 1);
    const int g = grid_for(N);
    switch (storage) {
        case TIPT_F64: stats_kernel<TIPT_F64><<<g, 256, 0, st>>>(field, labels, (int)nx, (int)ny, (int)nz, n_labels, s); break;
        case TIPT_F32: stats_kernel<TIPT_F32><<<g, 256, 0, st>>>(field, labels, (int)nx, (int)ny, (int)nz, n_labels, s); break;
        default: stats_kernel<TIPT_F32C><<<g, 256, 0, st>>>(field, labels, (int)nx, (int)ny, (int)nz, n_labels, s); break;
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "label statistics launch");
}
