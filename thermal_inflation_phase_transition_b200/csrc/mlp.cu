// Nucleation-rate surrogate network on the tensor cores (no reference
// counterpart: the reference measures nucleation only by running lattices).
//
// Network: 6 features (zero-padded to 16) -> 128 -> 128 -> 128 -> 17 outputs
// (zero-padded to 32), SiLU after the hidden layers.  Parameters are one FP32
// vector, per layer W[in][out] then b[out]; every kernel converts the weights
// it needs to BF16 in shared memory.  Matrix products take BF16 operands and
// accumulate in FP32 (mma.sync m16n8k16).
//
// One CTA owns a tile of 128 rows (8 warps x 16 rows) and carries it through
// every layer without leaving the SM: activations stay in shared memory, only
// the FP32 pre-activations of the hidden layers go to a global scratch for the
// backward pass of the same CTA.  The gradient kernel fuses forward, loss and
// backward; its per-tile parameter gradients go to a per-CTA slice of the
// workspace and a second kernel sums the slices in a fixed order, so training
// is deterministic.
//
// Loss per row (targets row: event, exposure, w_gamma, w_curve, f_1..f_16):
//   w_gamma (exp(l) exposure - event l) + w_curve/16 sum_k (softplus(o_k) - f_k o_k)
// with l = y[0] (clamped to [-40, 40] inside the exponential) the log rate in
// exposure units and o_k = y[k] the logits of the converted fraction at 16
// fixed times; the mean over `norm` rows is differentiated.
#include <cuda_bf16.h>

#include "tipt_internal.h"

namespace tipt {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int kRows = 128;     // rows per CTA tile
constexpr int kThreads = 256;  // 8 warps x 16 rows
constexpr int kWarps = kThreads / 32;
constexpr int kS = 136;        // shared row pitch (bf16): 68 words, conflict-free fragments
constexpr int kIn = 6;
constexpr int kOut = 17;
constexpr int kCurve = 16;
constexpr int kTgt = 4 + kCurve;
constexpr float kClamp = 40.0f;
constexpr int kBuf = 128 * kS;  // one shared operand buffer (bf16 elements)

__host__ __device__ constexpr int dim(int i) { return i == 0 ? 16 : (i == 4 ? 32 : 128); }
constexpr int w_off_rec(int l) {
    return l == 0 ? 0 : w_off_rec(l - 1) + dim(l - 1) * dim(l) + dim(l);
}
// offset of W_l (a select, so that a runtime layer index needs no call)
__host__ __device__ constexpr int w_off(int l) {
    return l == 0 ? 0 : l == 1 ? 2176 : l == 2 ? 18688 : l == 3 ? 35200 : 39328;
}
static_assert(w_off(1) == w_off_rec(1) && w_off(2) == w_off_rec(2) && w_off(3) == w_off_rec(3) &&
                  w_off(4) == w_off_rec(4),
              "layer offsets");
__host__ __device__ constexpr int b_off(int l) { return w_off(l) + dim(l) * dim(l + 1); }
constexpr int kParams = w_off(4);
static_assert(kParams == 39328, "parameter layout");

constexpr size_t kFwdSmem = 3 * kBuf * sizeof(bf16) + 128 * sizeof(float);
constexpr size_t kGradSmem = 4 * kBuf * sizeof(bf16) + (128 + kWarps * 128) * sizeof(float);

struct Args {
    const float* params;
    const float* x;       // [rows][6]
    const float* tgt;     // [rows][20]
    int64_t rows;
    float inv_norm;
    float* y;             // [rows][17] or nullptr
    float* zsave;         // [3][tiles*128][128]
    int64_t rows_pad;
    float* partials;      // [tiles][kParams]
    float* loss_rows;     // [rows] or nullptr
};

__device__ __forceinline__ uint32_t ld32(const bf16* p) {
    return *reinterpret_cast<const uint32_t*>(p);
}

__device__ __forceinline__ void st_pair(bf16* p, float a, float b) {
    *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(a, b);
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// c += A[m0:m0+16][0:K] * B[n0:n0+8][0:K]^T; both operands K-contiguous with pitch kS.
// Fragment ownership (PTX m16n8k16): lane = 4 g + t holds A rows g, g+8 at columns
// 2t, 2t+1, 2t+8, 2t+9, B column g at rows 2t, 2t+1, 2t+8, 2t+9, and C rows g, g+8
// at columns 2t, 2t+1.
__device__ __forceinline__ void tile_mma(const bf16* A, const bf16* B, int m0, int n0, int K,
                                         float c[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const bf16* a0 = A + (m0 + g) * kS + 2 * t;
    const bf16* a1 = a0 + 8 * kS;
    const bf16* b0 = B + (n0 + g) * kS + 2 * t;
#pragma unroll 4
    for (int k = 0; k < K; k += 16) {
        const uint32_t a[4] = {ld32(a0 + k), ld32(a1 + k), ld32(a0 + k + 8), ld32(a1 + k + 8)};
        const uint32_t b[2] = {ld32(b0 + k), ld32(b0 + k + 8)};
        mma_bf16(c, a, b);
    }
}

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigm(z);
    return s * (1.0f + z * (1.0f - s));
}

// W_l (FP32 [in][out]) -> bf16 [out][in] (forward operand B) or [in][out] (backward).
template <bool TRANSPOSED>
__device__ __forceinline__ void load_weights(const float* params, int l, bf16* Wb) {
    const int K = dim(l), N = dim(l + 1);
    const float* W = params + w_off(l);
    for (int e = threadIdx.x; e < K * N; e += kThreads) {
        const int i = e / N, o = e - i * N;
        const bf16 v = __float2bfloat16_rn(__ldg(W + e));
        if (TRANSPOSED) Wb[o * kS + i] = v;
        else Wb[i * kS + o] = v;
    }
}

// A warp's 16 x (8 NT) block of dZ (fragment layout) -> D (row-major), DT (transposed)
// and the warp's partial column sums of the FP32 values (fixed shuffle order).
template <int NT>
__device__ __forceinline__ void put_dz(const float (&v)[NT][4], bf16* D, bf16* DT, float* s_db) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int r0 = warp * 16 + g;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
        const int col = nt * 8 + 2 * t;
        st_pair(D + r0 * kS + col, v[nt][0], v[nt][1]);
        st_pair(D + (r0 + 8) * kS + col, v[nt][2], v[nt][3]);
        DT[col * kS + r0] = __float2bfloat16_rn(v[nt][0]);
        DT[(col + 1) * kS + r0] = __float2bfloat16_rn(v[nt][1]);
        DT[col * kS + r0 + 8] = __float2bfloat16_rn(v[nt][2]);
        DT[(col + 1) * kS + r0 + 8] = __float2bfloat16_rn(v[nt][3]);
        float s0 = v[nt][0] + v[nt][2], s1 = v[nt][1] + v[nt][3];
#pragma unroll
        for (int m = 4; m < 32; m <<= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, m);
            s1 += __shfl_xor_sync(0xffffffffu, s1, m);
        }
        if (g == 0) {
            s_db[warp * 128 + col] = s0;
            s_db[warp * 128 + col + 1] = s1;
        }
    }
}

template <bool GRAD>
__global__ void __launch_bounds__(kThreads) mlp_kernel(Args a) {
    extern __shared__ __align__(16) unsigned char smem[];
    bf16* Wb = reinterpret_cast<bf16*>(smem);
    bf16* B1 = Wb + kBuf;  // forward: layer input/output ping; backward: dZ (row-major)
    bf16* B2 = B1 + kBuf;  // forward: pong; backward: H^T
    bf16* B3 = B2 + kBuf;  // backward: dZ^T (gradient kernel only)
    float* s_bias = reinterpret_cast<float*>(smem + (GRAD ? 4 : 3) * kBuf * sizeof(bf16));
    float* s_db = s_bias + 128;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int rw = warp * 16;
    const int64_t row0 = (int64_t)blockIdx.x * kRows;

    // input tile, zero-padded to 16 features and to 128 rows
    for (int e = threadIdx.x; e < kRows * 16; e += kThreads) {
        const int r = e >> 4, c = e & 15;
        float v = 0.0f;
        if (c < kIn && row0 + r < a.rows) v = __ldg(a.x + (row0 + r) * kIn + c);
        B1[r * kS + c] = __float2bfloat16_rn(v);
    }
    bf16* hin = B1;
    bf16* hout = B2;
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int K = dim(l);
        __syncthreads();
        load_weights<true>(a.params, l, Wb);
        for (int e = threadIdx.x; e < 128; e += kThreads) s_bias[e] = __ldg(a.params + b_off(l) + e);
        __syncthreads();
#pragma unroll 1
        for (int nt = 0; nt < 16; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            tile_mma(hin, Wb, rw, nt * 8, K, c);
            const int col = nt * 8 + 2 * t;
            const float z0 = c[0] + s_bias[col], z1 = c[1] + s_bias[col + 1];
            const float z2 = c[2] + s_bias[col], z3 = c[3] + s_bias[col + 1];
            if (GRAD) {
                float* zs = a.zsave + ((int64_t)l * a.rows_pad + row0 + rw + g) * 128 + col;
                *reinterpret_cast<float2*>(zs) = make_float2(z0, z1);
                *reinterpret_cast<float2*>(zs + 8 * 128) = make_float2(z2, z3);
            }
            st_pair(hout + (rw + g) * kS + col, silu(z0), silu(z1));
            st_pair(hout + (rw + g + 8) * kS + col, silu(z2), silu(z3));
        }
        __syncwarp();
        bf16* tmp = hin;
        hin = hout;
        hout = tmp;
    }
    // output layer: 128 -> 32 (17 used); hin = B2
    __syncthreads();
    load_weights<true>(a.params, 3, Wb);
    for (int e = threadIdx.x; e < 32; e += kThreads) s_bias[e] = __ldg(a.params + b_off(3) + e);
    __syncthreads();
    float v[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        tile_mma(hin, Wb, rw, nt * 8, 128, c);
        const int col = nt * 8 + 2 * t;
        v[nt][0] = c[0] + s_bias[col];
        v[nt][1] = c[1] + s_bias[col + 1];
        v[nt][2] = c[2] + s_bias[col];
        v[nt][3] = c[3] + s_bias[col + 1];
    }
    if (a.y) {
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int col = nt * 8 + 2 * t + (q & 1);
                const int64_t row = row0 + rw + g + (q >> 1) * 8;
                if (col < kOut && row < a.rows) a.y[row * kOut + col] = v[nt][q];
            }
    }
    if constexpr (!GRAD) return;
    else {
        // loss and dL/dy per element; the gradient overwrites v
        float lsum[2] = {0.f, 0.f};
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int col = nt * 8 + 2 * t + (q & 1);
                const int64_t row = row0 + rw + g + (q >> 1) * 8;
                float d = 0.0f, loss = 0.0f;
                if (row < a.rows && col < kOut) {
                    const float* tg = a.tgt + row * kTgt;
                    const float yv = v[nt][q];
                    if (col == 0) {
                        const float ev = __ldg(tg), ex = __ldg(tg + 1), wg = __ldg(tg + 2);
                        const float E = expf(fminf(fmaxf(yv, -kClamp), kClamp));
                        loss = wg * (E * ex - ev * yv);
                        d = wg * ((fabsf(yv) < kClamp ? E : 0.0f) * ex - ev) * a.inv_norm;
                    } else {
                        const float wc = __ldg(tg + 3) * (1.0f / kCurve), f = __ldg(tg + 3 + col);
                        const float sp = fmaxf(yv, 0.0f) + log1pf(expf(-fabsf(yv)));
                        loss = wc * (sp - f * yv);
                        d = wc * (sigm(yv) - f) * a.inv_norm;
                    }
                }
                v[nt][q] = d;
                lsum[q >> 1] += loss;
            }
        if (a.loss_rows) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float s = lsum[h];
                s += __shfl_xor_sync(0xffffffffu, s, 1);
                s += __shfl_xor_sync(0xffffffffu, s, 2);
                const int64_t row = row0 + rw + g + h * 8;
                if (t == 0 && row < a.rows) a.loss_rows[row] = s;
            }
        }
        bf16* D = B1;   // free: layer 2 read B1, every warp passed the barrier above
        bf16* HT = B2;  // read by the output layer: rebuilt only after the next barrier
        bf16* DT = B3;
        put_dz<4>(v, D, DT, s_db);
        float* part = a.partials + (int64_t)blockIdx.x * kParams;
#pragma unroll
        for (int l = 3; l >= 0; --l) {
            const int K = dim(l), N = dim(l + 1);
            __syncthreads();
            for (int c = threadIdx.x; c < N; c += kThreads) {
                float s = 0.0f;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) s += s_db[w * 128 + c];
                part[b_off(l) + c] = s;
            }
            // H^T of this layer's input: the padded input tile or SiLU of the stored
            // pre-activations (rounded exactly as in the forward pass)
            for (int e = threadIdx.x; e < kRows * K; e += kThreads) {
                const int r = e / K, c = e - r * K;
                float hv;
                if (l == 0) hv = (c < kIn && row0 + r < a.rows) ? __ldg(a.x + (row0 + r) * kIn + c) : 0.0f;
                else hv = silu(a.zsave[((int64_t)(l - 1) * a.rows_pad + row0 + r) * 128 + c]);
                HT[c * kS + r] = __float2bfloat16_rn(hv);
            }
            if (l > 0) load_weights<false>(a.params, l, Wb);
            __syncthreads();
            // dW_l = H^T dZ over this tile's rows
            const int ntn = N / 8;
            for (int tile = warp; tile < (K / 16) * ntn; tile += kWarps) {
                const int mt = tile / ntn, nt = tile - mt * ntn;
                float c[4] = {0.f, 0.f, 0.f, 0.f};
                tile_mma(HT, DT, mt * 16, nt * 8, kRows, c);
                float* P = part + w_off(l) + (mt * 16 + g) * N + nt * 8 + 2 * t;
                *reinterpret_cast<float2*>(P) = make_float2(c[0], c[1]);
                *reinterpret_cast<float2*>(P + 8 * N) = make_float2(c[2], c[3]);
            }
            if (l == 0) break;
            // dZ_{l-1} = (dZ_l W_l^T) * SiLU'(z_{l-1}) for this warp's rows
            float u[16][4];
#pragma unroll
            for (int nt = 0; nt < 16; ++nt) {
                float c[4] = {0.f, 0.f, 0.f, 0.f};
                tile_mma(D, Wb, rw, nt * 8, N, c);
                const float* zs =
                    a.zsave + ((int64_t)(l - 1) * a.rows_pad + row0 + rw + g) * 128 + nt * 8 + 2 * t;
                const float2 za = *reinterpret_cast<const float2*>(zs);
                const float2 zb = *reinterpret_cast<const float2*>(zs + 8 * 128);
                u[nt][0] = c[0] * dsilu(za.x);
                u[nt][1] = c[1] * dsilu(za.y);
                u[nt][2] = c[2] * dsilu(zb.x);
                u[nt][3] = c[3] * dsilu(zb.y);
            }
            __syncthreads();  // every warp is done with DT, D and Wb of layer l
            put_dz<16>(u, D, DT, s_db);
        }
    }
}

// grad[p] = sum over tiles (fixed order, FP64 accumulation) of the per-tile slices.
__global__ void mlp_reduce_kernel(const float* part, int tiles, float* grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    double s = 0.0;
    for (int b = 0; b < tiles; ++b) s += (double)part[(int64_t)b * kParams + p];
    grad[p] = (float)s;
}

// Adam with bias correction (step t = *counter + offset + 1) and decoupled decay;
// the learning rate is lr x lr_sched[min(t, len) - 1] when a schedule is given.
__global__ void mlp_adam_kernel(float* p, const float* g, float* m, float* v,
                                const unsigned long long* ctr, long long offset, float lr,
                                const float* lr_sched, long long sched_len, float b1, float b2,
                                float eps, float wd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const long long t = (ctr ? (long long)*ctr : 0ll) + offset + 1;
    const double step = (double)t;
    if (lr_sched) lr *= lr_sched[(t < sched_len ? t : sched_len) - 1];
    const float bc1 = (float)(1.0 - pow((double)b1, step));
    const float bc2 = (float)(1.0 - pow((double)b2, step));
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i];
    p[i] = pi - lr * ((mi / bc1) / (sqrtf(vi / bc2) + eps) + wd * pi);
}

// ---------------------------------------------------------------- tcgen05 path
// The same network on the 5th-generation tensor cores.  Operands sit in shared
// memory in the canonical K-major, non-swizzled UMMA layout: a tile of R rows
// (the M or N extent) is stored as K/8 column chunks, each holding the R rows'
// 8 consecutive K values (16 bytes) back to back, so an 8 x 8 core matrix is 128
// contiguous bytes; descriptor LBO (next chunk along K) = 16 R bytes and SBO
// (next 8-row group) = 128 bytes.  Accumulators live in tensor memory: lane =
// tile row, column = output feature; one thread issues the MMAs and commits
// them to an mbarrier that every thread waits on with a time limit.  Warps w
// and w + 4 read the same 32 TMEM lanes (w % 4) and split the columns.
//
// Backward: dW = H^T dZ (M = in, N = out; for the 16-wide input layer
// dW^T = dZ^T H, M = out, N = 16) into TMEM columns [0, 128); dH = dZ W^T
// (M = rows, N = in) into columns [128, 256).

__device__ int g_mlp_status = 0;  // TIPT_ERR_TIMEOUT after a bounded wait expired
constexpr uint64_t kWaitNs = 2000000000ull;
constexpr int kTile = 128 * 128;  // bf16 elements of one operand buffer

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_test(bar, parity))
        if (global_ns() - t0 > kWaitNs) return false;
    return true;
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// element (r, k) of an R-row operand in the canonical layout
__device__ __forceinline__ int cidx(int r, int k, int R) { return (((k >> 3) * R + r) << 3) + (k & 7); }

// shared-memory matrix descriptor: start >> 4 in [0, 14), LBO >> 4 in [16, 30),
// SBO >> 4 in [32, 46), descriptor version 1 in [46, 48), no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, int R) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((R * 16) >> 4) << 16) |
           ((uint64_t)(128 >> 4) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B
// (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28
__host__ __device__ constexpr uint32_t idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}
// D[tmem] (+)= A(desc) B(desc)^T over one K = 16 step
__device__ __forceinline__ void umma(uint32_t d, uint64_t da, uint64_t db, uint32_t id,
                                     uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(da), "l"(db), "r"(id), "r"(acc));
}
// D = A[R_a rows][K] B[R_b rows][K]^T with K/16 instructions (issued by one thread)
__device__ __forceinline__ void gemm(uint32_t d, const bf16* A, int Ra, const bf16* B, int Rb,
                                     int K) {
    const uint32_t id = idesc(128, Rb);
    const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
    for (int kk = 0; kk < K / 16; ++kk)
        umma(d, sdesc(a0 + kk * 2 * Ra * 16, Ra), sdesc(b0 + kk * 2 * Rb * 16, Rb), id, kk > 0);
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
// 16 consecutive FP32 columns of this warp's 32 TMEM lanes (one row per thread)
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float (&f)[16]) {
    uint32_t v[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15])
        : "r"(addr));
    // the registers are valid only after the wait: tie them to it
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]),
                   "+r"(v[6]), "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]),
                   "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15])
                 :
                 : "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) f[j] = __uint_as_float(v[j]);
}
// 8 consecutive K values of one row -> one 16-byte store in the canonical layout
__device__ __forceinline__ void st_chunk(bf16* T, int r, int k0, int R, const float* f) {
    __nv_bfloat162 h[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) h[j] = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
    *reinterpret_cast<uint4*>(T + cidx(r, k0, R)) = *reinterpret_cast<uint4*>(h);
}
// sum over the warp's 32 rows of each of n columns, fixed butterfly order -> s[col]
template <int NC>
__device__ __forceinline__ void col_sums(const float* f, float* s, int c0) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        float v = f[j];
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
        if (lane == 0) s[c0 + j] = v;
    }
}

template <bool GRAD>
__global__ void __launch_bounds__(kThreads, 1) mlp_tc_kernel(Args a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    bf16* X0 = reinterpret_cast<bf16*>(sm);
    bf16* X1 = X0 + kTile;
    bf16* X2 = X1 + kTile;
    bf16* X3 = X2 + kTile;  // gradient kernel only
    float* s_bias = reinterpret_cast<float*>(X0 + (GRAD ? 4 : 3) * kTile);
    float* s_db = s_bias + 128;  // [4 lane quarters][128]
    uint64_t* bar = reinterpret_cast<uint64_t*>(s_db + 4 * 128);
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bar + 1);
    constexpr uint32_t kCols = GRAD ? 256 : 128;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int q = warp & 3, hf = warp >> 2;
    const int r = 32 * q + lane;  // tile row = TMEM lane read by this thread
    const int64_t row0 = (int64_t)blockIdx.x * kRows;
    const int64_t row = row0 + r;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(s_tmem)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 32) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // input tile, zero-padded to 16 features: thread = (row, 8-feature chunk)
    {
        const int rr = tid >> 1, c0 = (tid & 1) * 8;
        float f[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            f[j] = (c0 + j < kIn && row0 + rr < a.rows) ? __ldg(a.x + (row0 + rr) * kIn + c0 + j)
                                                         : 0.0f;
        st_chunk(X0, rr, c0, 128, f);
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = *s_tmem;
    const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16);  // this warp's lane quarter
    uint32_t phase = 0;
    bool ok = true;

    bf16* hin = X0;
    bf16* hout = X1;
#pragma unroll 1
    for (int l = 0; l < 4; ++l) {
        const int K = dim(l), N = dim(l + 1);
        // weights W_l -> X2 as B[N][K]
        const float* W = a.params + w_off(l);
        for (int e = tid; e < K * N; e += kThreads) {
            const int i = e / N, o = e - i * N;
            X2[cidx(o, i, N)] = __float2bfloat16_rn(__ldg(W + e));
        }
        if (tid < N) s_bias[tid] = __ldg(a.params + b_off(l) + tid);
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_after();
            gemm(tmem, hin, 128, X2, N, K);
            umma_commit(bar);
        }
        ok = mbar_wait(bar, phase);
        phase ^= 1u;
        if (!__syncthreads_and(ok)) goto done;
        tc_after();
        if (l < 3) {
#pragma unroll 1
            for (int c0 = 64 * hf; c0 < 64 * hf + 64; c0 += 16) {
                float z[16];
                tmem_ld16(tl + c0, z);
#pragma unroll
                for (int j = 0; j < 16; ++j) z[j] += s_bias[c0 + j];
                if (GRAD) {
                    float4* zs = reinterpret_cast<float4*>(
                        a.zsave + ((int64_t)l * a.rows_pad + row) * 128 + c0);
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        zs[j] = make_float4(z[4 * j], z[4 * j + 1], z[4 * j + 2], z[4 * j + 3]);
                }
#pragma unroll
                for (int j = 0; j < 16; ++j) z[j] = silu(z[j]);
                st_chunk(hout, r, c0, 128, z);
                st_chunk(hout, r, c0 + 8, 128, z + 8);
            }
            bf16* t = hin;
            hin = hout;
            hout = t;
        } else if (hf == 0) {
            // output layer: this thread holds row r's 32 outputs
            float y[32];
            tmem_ld16(tl, *reinterpret_cast<float(*)[16]>(y));
            tmem_ld16(tl + 16, *reinterpret_cast<float(*)[16]>(y + 16));
#pragma unroll
            for (int j = 0; j < 32; ++j) y[j] += s_bias[j];
            if (a.y && row < a.rows)
#pragma unroll
                for (int j = 0; j < kOut; ++j) a.y[row * kOut + j] = y[j];
            if (GRAD) {
                float loss = 0.0f;
                const bool valid = row < a.rows;
                const float* tg = a.tgt + (valid ? row : 0) * kTgt;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    float d = 0.0f;
                    if (valid && j < kOut) {
                        const float yv = y[j];
                        if (j == 0) {
                            const float ev = __ldg(tg), ex = __ldg(tg + 1), wg = __ldg(tg + 2);
                            const float E = expf(fminf(fmaxf(yv, -kClamp), kClamp));
                            loss += wg * (E * ex - ev * yv);
                            d = wg * ((fabsf(yv) < kClamp ? E : 0.0f) * ex - ev) * a.inv_norm;
                        } else {
                            const float wc = __ldg(tg + 3) * (1.0f / kCurve), f = __ldg(tg + 3 + j);
                            const float sp = fmaxf(yv, 0.0f) + log1pf(expf(-fabsf(yv)));
                            loss += wc * (sp - f * yv);
                            d = wc * (sigm(yv) - f) * a.inv_norm;
                        }
                    }
                    y[j] = d;
                }
                if (a.loss_rows && valid) a.loss_rows[row] = loss;
                // dZ of the output layer: D = X0 [128 rows][32], DT = X3 [32][128 rows]
#pragma unroll
                for (int c0 = 0; c0 < 32; c0 += 8) st_chunk(X0, r, c0, 128, y + c0);
#pragma unroll
                for (int j = 0; j < 32; ++j) X3[cidx(j, r, 32)] = __float2bfloat16_rn(y[j]);
                col_sums<32>(y, s_db + q * 128, 0);
            }
        }
        tc_before();
        fence_async_smem();
        __syncthreads();
    }
    if constexpr (GRAD) {
        float* part = a.partials + (int64_t)blockIdx.x * kParams;
        bf16* D = X0;
        bf16* HT = X1;
        bf16* Wb = X2;
        bf16* DT = X3;
#pragma unroll 1
        for (int l = 3; l >= 0; --l) {
            const int K = dim(l), N = dim(l + 1);
            if (tid < N) part[b_off(l) + tid] = ((s_db[tid] + s_db[128 + tid]) + s_db[256 + tid]) +
                                                s_db[384 + tid];
            // H^T of this layer's input: [K rows][128 tile rows]
            for (int e = tid; e < 128 * K; e += kThreads) {
                const int rr = e / K, c = e - rr * K;
                float hv;
                if (l == 0) hv = (c < kIn && row0 + rr < a.rows) ? __ldg(a.x + (row0 + rr) * kIn + c) : 0.0f;
                else hv = silu(a.zsave[((int64_t)(l - 1) * a.rows_pad + row0 + rr) * 128 + c]);
                HT[cidx(c, rr, K)] = __float2bfloat16_rn(hv);
            }
            if (l > 0) {
                const float* W = a.params + w_off(l);
                for (int e = tid; e < K * N; e += kThreads) {
                    const int i = e / N, o = e - i * N;
                    Wb[cidx(i, o, 128)] = __float2bfloat16_rn(__ldg(W + e));
                }
            }
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc_after();
                if (l > 0) {
                    gemm(tmem, HT, 128, DT, N, 128);       // dW[in][out]
                    gemm(tmem + 128, D, 128, Wb, 128, N);  // dH[rows][in]
                } else {
                    gemm(tmem, DT, 128, HT, 16, 128);      // dW^T[out][in]
                }
                umma_commit(bar);
            }
            ok = mbar_wait(bar, phase);
            phase ^= 1u;
            if (!__syncthreads_and(ok)) goto done;
            tc_after();
            if (l > 0) {
                // dW rows i = r, this half's output columns
                const int nh = N / 2;
#pragma unroll 1
                for (int c0 = hf * nh; c0 < hf * nh + nh; c0 += 16) {
                    float g[16];
                    tmem_ld16(tl + c0, g);
                    float4* P = reinterpret_cast<float4*>(part + w_off(l) + r * N + c0);
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        P[j] = make_float4(g[4 * j], g[4 * j + 1], g[4 * j + 2], g[4 * j + 3]);
                }
                // dZ_{l-1} = dH * SiLU'(z_{l-1}) for row r, this half's 64 input columns
#pragma unroll 1
                for (int c0 = 64 * hf; c0 < 64 * hf + 64; c0 += 16) {
                    float g[16];
                    tmem_ld16(tl + 128 + c0, g);
                    const float4* zs = reinterpret_cast<const float4*>(
                        a.zsave + ((int64_t)(l - 1) * a.rows_pad + row) * 128 + c0);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float4 z = zs[j];
                        g[4 * j] *= dsilu(z.x);
                        g[4 * j + 1] *= dsilu(z.y);
                        g[4 * j + 2] *= dsilu(z.z);
                        g[4 * j + 3] *= dsilu(z.w);
                    }
                    st_chunk(D, r, c0, 128, g);
                    st_chunk(D, r, c0 + 8, 128, g + 8);
#pragma unroll
                    for (int j = 0; j < 16; ++j) DT[cidx(c0 + j, r, 128)] = __float2bfloat16_rn(g[j]);
                    col_sums<16>(g, s_db + q * 128, c0);
                }
            } else if (hf == 0) {
                // dW^T rows o = r, 16 input columns
                float g[16];
                tmem_ld16(tl, g);
#pragma unroll
                for (int j = 0; j < 16; ++j) part[w_off(0) + j * 128 + r] = g[j];
            }
            tc_before();
            fence_async_smem();
            __syncthreads();
        }
    }
done:
    if (!ok && tid == 0) atomicExch(&g_mlp_status, (int)TIPT_ERR_TIMEOUT);
    tc_before();
    __syncthreads();
    if (warp == 0) {
        tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols)
                     : "memory");
    }
}

constexpr size_t kTcFwdSmem = 3 * kTile * sizeof(bf16) + (128 + 512) * sizeof(float) + 16 + 1024;
constexpr size_t kTcGradSmem = 4 * kTile * sizeof(bf16) + (128 + 512) * sizeof(float) + 16 + 1024;

int g_policy = 0;  // 0 automatic (tcgen05), 1 mma.sync, 2 tcgen05

int64_t tiles_of(int64_t rows) { return (rows + kRows - 1) / kRows; }

int64_t workspace_bytes(int64_t rows) {
    const int64_t tiles = tiles_of(rows);
    return (3 * tiles * kRows * 128 + tiles * (int64_t)kParams) * (int64_t)sizeof(float);
}

int check_rows(int64_t rows) {
    if (rows < 1 || rows > (1ll << 24))
        return fail(TIPT_ERR_ARG, "rows must be in [1, 2^24], got %lld", (long long)rows);
    return TIPT_OK;
}

}  // namespace mlp

// Read (and optionally clear) the surrogate kernels' status word.
int mlp_status(int* status, int clear) {
    cudaError_t e = cudaMemcpyFromSymbol(status, mlp::g_mlp_status, sizeof(int));
    if (e == cudaSuccess && clear) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(mlp::g_mlp_status, &zero, sizeof(int));
    }
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "mlp status");
}

}  // namespace tipt

using namespace tipt;
using namespace tipt::mlp;

extern "C" int tipt_mlp_set_policy(int policy) {
    if (policy < 0 || policy > 2) return fail(TIPT_ERR_ARG, "policy must be 0, 1 or 2");
    g_policy = policy;
    return TIPT_OK;
}

extern "C" int64_t tipt_mlp_param_count(void) { return kParams; }

extern "C" int64_t tipt_mlp_workspace_size(int64_t rows) {
    return rows < 1 ? 0 : mlp::workspace_bytes(rows);
}

extern "C" int tipt_mlp_forward(const float* params, const float* x, int64_t rows, float* y,
                                void* stream) {
    int rc;
    if ((rc = check_rows(rows)) || (rc = check_ptr(params, 4, "params")) ||
        (rc = check_ptr(x, 4, "x")) || (rc = check_ptr(y, 4, "y")))
        return rc;
    Args a{};
    a.params = params;
    a.x = x;
    a.rows = rows;
    a.y = y;
    cudaError_t e;
    if (g_policy == 1) {
        e = cudaFuncSetAttribute(mlp_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kFwdSmem);
        if (e != cudaSuccess) return fail_cuda(e, "mlp forward attributes");
        mlp_kernel<false><<<(unsigned)tiles_of(rows), kThreads, kFwdSmem, (cudaStream_t)stream>>>(a);
    } else {
        e = cudaFuncSetAttribute(mlp_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kTcFwdSmem);
        if (e != cudaSuccess) return fail_cuda(e, "mlp forward attributes");
        mlp_tc_kernel<false>
            <<<(unsigned)tiles_of(rows), kThreads, kTcFwdSmem, (cudaStream_t)stream>>>(a);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "mlp forward launch");
}

extern "C" int tipt_mlp_grad(const float* params, const float* x, const float* tgt, int64_t rows,
                             float norm, float* grad, float* loss_rows, void* workspace,
                             int64_t workspace_bytes, void* stream) {
    int rc;
    if ((rc = check_rows(rows)) || (rc = check_ptr(params, 4, "params")) ||
        (rc = check_ptr(x, 4, "x")) || (rc = check_ptr(tgt, 4, "tgt")) ||
        (rc = check_ptr(grad, 4, "grad")) || (rc = check_ptr(workspace, 16, "workspace")))
        return rc;
    if (!(norm > 0.0f)) return fail(TIPT_ERR_ARG, "norm must be > 0");
    const int64_t need = mlp::workspace_bytes(rows);
    if (workspace_bytes < need)
        return fail(TIPT_ERR_ARG, "workspace of %lld bytes is smaller than the %lld needed",
                    (long long)workspace_bytes, (long long)need);
    const int64_t tiles = tiles_of(rows);
    Args a{};
    a.params = params;
    a.x = x;
    a.tgt = tgt;
    a.rows = rows;
    a.inv_norm = 1.0f / norm;
    a.zsave = static_cast<float*>(workspace);
    a.rows_pad = tiles * kRows;
    a.partials = a.zsave + 3 * a.rows_pad * 128;
    a.loss_rows = loss_rows;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if (g_policy == 1) {
        e = cudaFuncSetAttribute(mlp_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kGradSmem);
        if (e != cudaSuccess) return fail_cuda(e, "mlp gradient attributes");
        mlp_kernel<true><<<(unsigned)tiles, kThreads, kGradSmem, st>>>(a);
    } else {
        e = cudaFuncSetAttribute(mlp_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kTcGradSmem);
        if (e != cudaSuccess) return fail_cuda(e, "mlp gradient attributes");
        mlp_tc_kernel<true><<<(unsigned)tiles, kThreads, kTcGradSmem, st>>>(a);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "mlp gradient launch");
    mlp_reduce_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(a.partials, (int)tiles, grad);
    e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "mlp gradient reduce launch");
}

extern "C" int tipt_mlp_adam(float* params, const float* grad, float* m, float* v,
                             const uint64_t* counter, int64_t offset, float lr,
                             const float* lr_schedule, int64_t schedule_len, float beta1,
                             float beta2, float eps, float weight_decay, void* stream) {
    int rc;
    if ((rc = check_ptr(params, 4, "params")) || (rc = check_ptr(grad, 4, "grad")) ||
        (rc = check_ptr(m, 4, "m")) || (rc = check_ptr(v, 4, "v")))
        return rc;
    if (counter && (rc = check_ptr(counter, 8, "counter"))) return rc;
    if (lr_schedule && ((rc = check_ptr(lr_schedule, 4, "lr_schedule")) || schedule_len < 1))
        return rc ? rc : fail(TIPT_ERR_ARG, "schedule_len must be >= 1");
    if (offset < 0) return fail(TIPT_ERR_ARG, "offset must be >= 0");
    mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        params, grad, m, v, reinterpret_cast<const unsigned long long*>(counter), (long long)offset,
        lr, lr_schedule, (long long)schedule_len, beta1, beta2, eps, weight_decay);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TIPT_OK : fail_cuda(e, "mlp adam launch");
}
