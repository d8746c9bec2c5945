// rq_mlp.cu -- BF16 tensor-core (tcgen05) GEMMs and the warm-start MLP.
//
// The warm start for QAOA angles is a small MLP (325 -> 256 -> 256 -> 8, ReLU,
// BF16 weights and activations, FP32 accumulation).  It has no counterpart in
// the reference (whose run_qaoa always starts from gamma = beta = 0.5,
// qaoa.rs:221-222); it is trained on angles the batched simulator optimises.
//
// k_gemm_bf16 computes C[M x N] = A[M x K] * B[N x K]^T (+ epilogue) on the
// 5th-generation tensor cores: each CTA owns a 128-row tile of C and up to 256
// columns; K is consumed in chunks of 64.  Operands are copied from global
// memory into shared memory in the no-swizzle K-major "core matrix" layout
// (8 rows x 16 bytes per core matrix; element (r, k) of a tile at byte
// (r/8)*SBO + (k/8)*LBO + (r%8)*16 + (k%8)*2 with LBO = 128, SBO = 1024),
// one elected thread issues tcgen05.mma (kind::f16, BF16 inputs, FP32
// accumulator in tensor memory), tcgen05.commit signals an mbarrier, and the
// epilogue reads the accumulator back with tcgen05.ld.  Every wait on the
// mbarrier is bounded; on expiry the kernel records an error and returns after
// freeing its tensor memory.
#include "rq_internal.cuh"

#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

constexpr int BM = 128;      // rows per CTA (UMMA M)
constexpr int BK = 64;       // K per shared-memory chunk
constexpr int LBO = 128;     // bytes between core matrices along K
constexpr int SBO = (BK / 8) * 128;   // bytes between 8-row groups

__device__ int g_mma_timeout = 0;   // set when a bounded wait expires

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor, no swizzle, K-major (sm_100 version 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)(LBO >> 4) << 16;
    d |= (uint64_t)(SBO >> 4) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for sm_100
    return d;                 // base offset 0, lbo mode 0, layout type 0 (no swizzle)
}

// instruction descriptor: BF16 x BF16 -> F32, A and B K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4)               // D format F32
         | (1u << 7)               // A format BF16
         | (1u << 10)              // B format BF16
         | ((uint32_t)(n >> 3) << 17)
         | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// polls before a main-path wait counts as expired (rq_debug_set_wait_limit); the clean-up
// wait after an expiry always uses WAIT_POLLS
constexpr uint32_t WAIT_POLLS = 1u << 26;
__device__ uint32_t g_mma_wait_polls = WAIT_POLLS;

// bounded wait for the mbarrier phase `parity`; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t polls = WAIT_POLLS) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < polls; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

enum Epi : int {
    EPI_F32 = 0,         // C (f32) = acc
    EPI_BIAS_RELU = 1,   // Z (f32) = acc + bias; H (bf16) = relu(Z)
    EPI_BIAS = 2         // C (f32) = acc + bias
};

struct GemmArgs {
    const __nv_bfloat16* A;   // [M x K] row-major
    const __nv_bfloat16* B;   // [N x K] row-major
    int M, N, K;              // M % 128 == 0, N % 16 == 0, K % 16 == 0
    int lda, ldb;             // row strides (elements)
    float* C;                 // [M x N] f32 (row stride ldc)
    int ldc;
    const float* bias;        // [N]
    __nv_bfloat16* H;         // [M x N] bf16 (row stride ldh), EPI_BIAS_RELU
    int ldh;
    int epi;
};

// Tile of C: rows [blockIdx.x*128, +128), cols [blockIdx.y*NT, +NT).  128 threads.
template <int NT>
__global__ void __launch_bounds__(128, 1) k_gemm_bf16(GemmArgs g) {
    static_assert(NT % 16 == 0 && NT >= 32 && NT <= 256, "tile N");
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem;                        // 128 x 64 bf16 = 16 KB
    unsigned char* sB = smem + BM * BK * 2;          // NT x 64 bf16
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int timed_out;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int row0 = blockIdx.x * BM, col0 = blockIdx.y * NT;
    const int ncols = NT < 32 ? 32 : NT;   // tensor-memory columns (power of two >= 32)

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        timed_out = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    const int nk = g.K / BK + ((g.K % BK) ? 1 : 0);
    uint32_t phase = 0;
    for (int kc = 0; kc < nk; ++kc) {
        const int k0 = kc * BK;
        const int kw = min(BK, g.K - k0);   // multiple of 16
        // stage A (128 x kw) and B (NT x kw) into the core-matrix layout, 16 bytes per access
        const int chunksA = BM * (kw / 8), chunksB = NT * (kw / 8);
        for (int c = tid; c < chunksA + chunksB; c += blockDim.x) {
            const bool isA = c < chunksA;
            const int cc = isA ? c : c - chunksA;
            const int r = cc / (kw / 8), kk = (cc % (kw / 8)) * 8;
            const int grow = isA ? row0 + r : col0 + r;   // rows past M / N read as zeros
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (grow < (isA ? g.M : g.N)) {
                const __nv_bfloat16* src = isA ? g.A + (size_t)grow * g.lda + k0 + kk : g.B + (size_t)grow * g.ldb + k0 + kk;
                v = *reinterpret_cast<const uint4*>(src);
            }
            unsigned char* dst = (isA ? sA : sB) + (r >> 3) * SBO + (kk >> 3) * LBO + (r & 7) * 16;
            *reinterpret_cast<uint4*>(dst) = v;
        }
        // make the generic-proxy writes visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int ks = 0; ks < kw / 16; ++ks) {
                const uint64_t ad = sdesc(a0 + ks * 2 * LBO);
                const uint64_t bd = sdesc(b0 + ks * 2 * LBO);
                const uint32_t acc = (kc > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc_bf16(NT)), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mbar))
                         : "memory");
        }
        // the chunk's MMAs must finish before the buffers are overwritten (and before the epilogue)
        if (!mbar_wait(&mbar, phase, g_mma_wait_polls)) {
            timed_out = 1;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
        if (timed_out) {
            // the MMAs of this chunk may still be in flight: let them land (bounded) before the
            // shared and tensor memory they use are released
            if (tid == 0) mbar_wait(&mbar, phase ^ 1u);
            break;
        }
    }

    if (!timed_out) {
        // epilogue: warp w holds rows 32w..32w+31 in tensor-memory lanes 32w..
        const int r = row0 + warp * 32 + (tid & 31);
        for (int c0 = 0; c0 < NT; c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (r < g.M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int c = col0 + c0 + j;
                    if (c >= g.N) continue;
                    float x = __uint_as_float(v[j]);
                    if (g.epi != EPI_F32) x += g.bias[c];
                    g.C[(size_t)r * g.ldc + c] = x;
                    if (g.epi == EPI_BIAS_RELU) g.H[(size_t)r * g.ldh + c] = __float2bfloat16_rn(x > 0.f ? x : 0.f);
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(&g_mma_timeout, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

}  // namespace

namespace rq {

// C = A * B^T with the given epilogue, on `stream`.  Shapes are checked here.
int gemm_bf16(cudaStream_t stream, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N,
              int K, float* C, int ldc, int epi, const float* bias, __nv_bfloat16* H, int ldh) {
    if (M < 1 || N < 1 || K < 16 || K % 16)
        return fail(RQ_ERR_INVALID_ARGUMENT, "gemm_bf16: M, N >= 1 and K a positive multiple of 16");
    if (lda % 8 || ldb % 8) return fail(RQ_ERR_INVALID_ARGUMENT, "gemm_bf16: row strides must be multiples of 8");
    GemmArgs g{A, B, M, N, K, lda, ldb, C, ldc, bias, H, ldh, epi};
    const int nt = N > 128 ? 256 : (N > 64 ? 128 : (N > 32 ? 64 : 32));
    dim3 grid((M + BM - 1) / BM, (N + nt - 1) / nt);
    const size_t smem = (size_t)(BM + nt) * BK * 2;
    switch (nt) {
        case 256:
            RQ_CUDA(cudaFuncSetAttribute(k_gemm_bf16<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_gemm_bf16<256><<<grid, 128, smem, stream>>>(g);
            break;
        case 128:
            RQ_CUDA(cudaFuncSetAttribute(k_gemm_bf16<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_gemm_bf16<128><<<grid, 128, smem, stream>>>(g);
            break;
        case 64:
            RQ_CUDA(cudaFuncSetAttribute(k_gemm_bf16<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_gemm_bf16<64><<<grid, 128, smem, stream>>>(g);
            break;
        default:
            RQ_CUDA(cudaFuncSetAttribute(k_gemm_bf16<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_gemm_bf16<32><<<grid, 128, smem, stream>>>(g);
            break;
    }
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

int mma_timeout_flag(int* out) {
    int v = 0, zero = 0;
    RQ_CUDA(cudaMemcpyFromSymbol(&v, g_mma_timeout, sizeof(int)));
    if (v) {
        RQ_CUDA(cudaMemcpyToSymbol(g_mma_timeout, &zero, sizeof(int)));
        RQ_CUDA(cudaDeviceSynchronize());
    }
    *out = v;
    return RQ_OK;
}

int mma_set_wait_polls(uint32_t polls) {
    const uint32_t v = polls == RQ_WAIT_LIMIT_DEFAULT ? WAIT_POLLS : polls;
    RQ_CUDA(cudaMemcpyToSymbol(g_mma_wait_polls, &v, sizeof(v)));
    RQ_CUDA(cudaDeviceSynchronize());   // landed before any later launch, on any stream
    return RQ_OK;
}

}  // namespace rq

extern "C" {

// C (f32, M x N) = A (bf16, M x K) * B (bf16, N x K)^T on the tensor cores;
// host buffers in and out (test and benchmark entry point of the GEMM).
int rq_gemm_bf16(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K, float* C) {
    if (!A || !B || !C) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float* dC = nullptr;
    RQ_CUDA(cudaMalloc(&dA, (size_t)M * K * 2));
    RQ_CUDA(cudaMalloc(&dB, (size_t)N * K * 2));
    RQ_CUDA(cudaMalloc(&dC, (size_t)M * N * 4));
    int rc = RQ_OK;
    cudaError_t e = cudaMemcpy(dA, A, (size_t)M * K * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dB, B, (size_t)N * K * 2, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = rq::cuda_fail(e, "cudaMemcpy");
    if (rc == RQ_OK) rc = rq::gemm_bf16(0, dA, K, dB, K, M, N, K, dC, N, EPI_F32, nullptr, nullptr, 0);
    if (rc == RQ_OK) {
        e = cudaMemcpy(C, dC, (size_t)M * N * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = rq::cuda_fail(e, "cudaMemcpy");
    }
    int to = 0;
    if (rc == RQ_OK && rq::mma_timeout_flag(&to) == RQ_OK && to)
        rc = rq::fail(RQ_ERR_TIMEOUT, "tensor-core wait expired");
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    return rc;
}

}  // extern "C"

// ===========================================================================
// The warm-start MLP: in -> h1 -> h2 -> out, ReLU after the two hidden layers,
// FP32 master parameters (row-major [out_features x in_features] weights and
// biases), BF16 copies for the tensor-core GEMMs, FP32 accumulation, mean
// squared error loss, Adam updates in FP32 on the device.
// ===========================================================================
namespace {

__global__ void k_pad_bf16(const float* __restrict__ src, int rows, int cols, int lds, __nv_bfloat16* __restrict__ dst,
                           int prow, int pcol, int ldd) {
    const long total = (long)prow * pcol;
    for (long w = (long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (long)gridDim.x * blockDim.x) {
        const int r = (int)(w / pcol), c = (int)(w - (long)r * pcol);
        const float v = (r < rows && c < cols) ? src[(long)r * lds + c] : 0.f;
        dst[(long)r * ldd + c] = __float2bfloat16_rn(v);
    }
}

// dst[c][r] = src[r][c]  (rows x cols -> cols x rows)
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ src, int rows, int cols, int lds,
                                 __nv_bfloat16* __restrict__ dst, int ldd) {
    __shared__ __nv_bfloat16 t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        t[j][threadIdx.x] = (r < rows && c < cols) ? src[(long)r * lds + c] : __float2bfloat16_rn(0.f);
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = bx + j, r = by + threadIdx.x;
        if (c < cols && r < rows) dst[(long)c * ldd + r] = t[threadIdx.x][j];
    }
}

// MSE over the valid B x out block; dY (bf16, Bp x ldy) = 2 (Y - T) / (B out); db = column sums of dY (f32)
__global__ void k_mse_grad(const float* __restrict__ Y, int ldy, const float* __restrict__ T, int B, int out,
                           __nv_bfloat16* __restrict__ dY, int Bp, int outp, float* __restrict__ db,
                           float* __restrict__ loss) {
    __shared__ float red[32];
    const float inv = 1.f / (float)(B * out);
    float l = 0.f;
    for (int w = threadIdx.x; w < Bp * outp; w += blockDim.x) {
        const int r = w / outp, c = w - r * outp;
        float g = 0.f;
        if (r < B && c < out) {
            const float d = Y[(long)r * ldy + c] - T[(long)r * out + c];
            l += d * d;
            g = 2.f * d * inv;
        }
        dY[(long)r * outp + c] = __float2bfloat16_rn(g);
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
        *loss = s * inv;
    }
    // bias gradient of the output layer (same scaling as dY)
    for (int c = threadIdx.x; c < out; c += blockDim.x) {
        float s = 0.f;
        for (int r = 0; r < B; ++r) s += 2.f * (Y[(long)r * ldy + c] - T[(long)r * out + c]) * inv;
        db[c] = s;
    }
}

// dZ = dH * (Z > 0) (bf16, rows >= B zeroed); db[c] = sum over the B valid rows
__global__ void k_relu_back(const float* __restrict__ dH, const float* __restrict__ Z, int B, int Bp, int cols,
                            __nv_bfloat16* __restrict__ dZ, float* __restrict__ db) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int r = 0; r < Bp; ++r) {
            float g = 0.f;
            if (r < B) {
                g = Z[(long)r * cols + c] > 0.f ? dH[(long)r * cols + c] : 0.f;
                s += g;
            }
            dZ[(long)r * cols + c] = __float2bfloat16_rn(g);
        }
        db[c] = s;
    }
}

// Adam on a [rows x cols] parameter block whose gradient sits at g[(r * gsr) + c * gsc]
__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                       int rows, int cols, long gsr, long gsc, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    const long total = (long)rows * cols;
    for (long w = (long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (long)gridDim.x * blockDim.x) {
        const long r = w / cols, c = w - r * cols;
        const float gr = g[r * gsr + c * gsc];
        const float mm = b1 * m[w] + (1.f - b1) * gr;
        const float vv = b2 * v[w] + (1.f - b2) * gr * gr;
        m[w] = mm;
        v[w] = vv;
        p[w] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

// gradient block copy into the caller's flat layout
__global__ void k_gather(const float* __restrict__ g, int rows, int cols, long gsr, long gsc, float* __restrict__ out) {
    const long total = (long)rows * cols;
    for (long w = (long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (long)gridDim.x * blockDim.x) {
        const long r = w / cols, c = w - r * cols;
        out[w] = g[r * gsr + c * gsc];
    }
}

inline int pad16(int x) { return (x + 15) & ~15; }

}  // namespace

struct rq_mlp {
    int device = 0;
    int in = 0, h1 = 0, h2 = 0, out = 0;
    int inp = 0, outp = 0;        // padded widths (K multiple of 16, N padded to 32)
    cudaStream_t stream = nullptr;
    // FP32 master parameters and Adam moments, one flat buffer each
    float *P = nullptr, *Mo = nullptr, *Vo = nullptr;
    long off_w1 = 0, off_b1 = 0, off_w2 = 0, off_b2 = 0, off_w3 = 0, off_b3 = 0, nparam = 0;
    long step = 0;
    // BF16 copies: W1b [h1 x inp], W2b [h2 x h1], W3b [outp x h2], W2t [h1 x h2], W3t [h2 x outp]
    __nv_bfloat16 *W1b = nullptr, *W2b = nullptr, *W3b = nullptr, *W2t = nullptr, *W3t = nullptr;
    // batch workspace
    int cap = 0;
    __nv_bfloat16 *X = nullptr, *Xt = nullptr, *H1 = nullptr, *H1t = nullptr, *H2 = nullptr, *H2t = nullptr;
    __nv_bfloat16 *dY = nullptr, *dYt = nullptr, *dZ2 = nullptr, *dZ2t = nullptr, *dZ1 = nullptr, *dZ1t = nullptr;
    float *Xf = nullptr, *Tf = nullptr, *Z1 = nullptr, *Z2 = nullptr, *Y = nullptr, *dH2 = nullptr, *dH1 = nullptr;
    float *G = nullptr;           // gradients: dW1 [h1 x inp], db1, dW2 [h2 x h1], db2, dW3t [h2 x outp], db3
    long g_w1 = 0, g_b1 = 0, g_w2 = 0, g_b2 = 0, g_w3t = 0, g_b3 = 0, g_total = 0;
    float* loss = nullptr;
};

namespace {

template <typename P>
int dalloc(P** p, size_t n) {
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(1, n) * sizeof(P));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return rq::fail(RQ_ERR_MEMORY_ALLOCATION, "memory allocation failed: need " + std::to_string(n * sizeof(P)) + " bytes");
    }
    return RQ_OK;
}

int mlp_refresh_bf16(rq_mlp* m) {
    const int sms = rq::num_sms(m->device);
    const float* P = m->P;
    k_pad_bf16<<<rq::grid_for((uint64_t)m->h1 * m->inp, 256, sms), 256, 0, m->stream>>>(P + m->off_w1, m->h1, m->in, m->in,
                                                                                     m->W1b, m->h1, m->inp, m->inp);
    k_pad_bf16<<<rq::grid_for((uint64_t)m->h2 * m->h1, 256, sms), 256, 0, m->stream>>>(P + m->off_w2, m->h2, m->h1, m->h1,
                                                                                    m->W2b, m->h2, m->h1, m->h1);
    k_pad_bf16<<<rq::grid_for((uint64_t)m->outp * m->h2, 256, sms), 256, 0, m->stream>>>(P + m->off_w3, m->out, m->h2,
                                                                                      m->h2, m->W3b, m->outp, m->h2, m->h2);
    dim3 tb(32, 8);
    k_transpose_bf16<<<dim3((m->h1 + 31) / 32, (m->h2 + 31) / 32), tb, 0, m->stream>>>(m->W2b, m->h2, m->h1, m->h1, m->W2t,
                                                                                       m->h2);
    k_transpose_bf16<<<dim3((m->h2 + 31) / 32, (m->outp + 31) / 32), tb, 0, m->stream>>>(m->W3b, m->outp, m->h2, m->h2,
                                                                                         m->W3t, m->outp);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

int mlp_reserve(rq_mlp* m, int B) {
    const int Bp = (B + 127) & ~127;
    if (Bp <= m->cap) return RQ_OK;
    void* bufs[] = {m->X, m->Xt, m->H1, m->H1t, m->H2, m->H2t, m->dY, m->dYt, m->dZ2, m->dZ2t, m->dZ1, m->dZ1t,
                    m->Xf, m->Tf, m->Z1, m->Z2, m->Y, m->dH2, m->dH1};
    for (void* b : bufs) if (b) cudaFree(b);
    const size_t b = (size_t)Bp;
    RQ_TRY(dalloc(&m->X, b * m->inp));
    RQ_TRY(dalloc(&m->Xt, b * m->inp));
    RQ_TRY(dalloc(&m->H1, b * m->h1));
    RQ_TRY(dalloc(&m->H1t, b * m->h1));
    RQ_TRY(dalloc(&m->H2, b * m->h2));
    RQ_TRY(dalloc(&m->H2t, b * m->h2));
    RQ_TRY(dalloc(&m->dY, b * m->outp));
    RQ_TRY(dalloc(&m->dYt, b * m->outp));
    RQ_TRY(dalloc(&m->dZ2, b * m->h2));
    RQ_TRY(dalloc(&m->dZ2t, b * m->h2));
    RQ_TRY(dalloc(&m->dZ1, b * m->h1));
    RQ_TRY(dalloc(&m->dZ1t, b * m->h1));
    RQ_TRY(dalloc(&m->Xf, b * m->in));
    RQ_TRY(dalloc(&m->Tf, b * m->out));
    RQ_TRY(dalloc(&m->Z1, b * m->h1));
    RQ_TRY(dalloc(&m->Z2, b * m->h2));
    RQ_TRY(dalloc(&m->Y, b * m->outp));
    RQ_TRY(dalloc(&m->dH2, b * m->h2));
    RQ_TRY(dalloc(&m->dH1, b * m->h1));
    m->cap = Bp;
    return RQ_OK;
}

// forward on m->Xf (B x in, f32 on device): Z1, H1, Z2, H2, Y
int mlp_forward_dev(rq_mlp* m, int B) {
    const int Bp = (B + 127) & ~127;
    const int sms = rq::num_sms(m->device);
    k_pad_bf16<<<rq::grid_for((uint64_t)Bp * m->inp, 256, sms), 256, 0, m->stream>>>(m->Xf, B, m->in, m->in, m->X, Bp,
                                                                                  m->inp, m->inp);
    RQ_CUDA(cudaGetLastError());
    RQ_TRY(rq::gemm_bf16(m->stream, m->X, m->inp, m->W1b, m->inp, Bp, m->h1, m->inp, m->Z1, m->h1, EPI_BIAS_RELU,
                         m->P + m->off_b1, m->H1, m->h1));
    RQ_TRY(rq::gemm_bf16(m->stream, m->H1, m->h1, m->W2b, m->h1, Bp, m->h2, m->h1, m->Z2, m->h2, EPI_BIAS_RELU,
                         m->P + m->off_b2, m->H2, m->h2));
    RQ_TRY(rq::gemm_bf16(m->stream, m->H2, m->h2, m->W3b, m->h2, Bp, m->out, m->h2, m->Y, m->outp, EPI_BIAS,
                         m->P + m->off_b3, nullptr, 0));
    return RQ_OK;
}

// backward after mlp_forward_dev with targets in m->Tf: gradients into m->G, loss into m->loss
int mlp_backward_dev(rq_mlp* m, int B) {
    const int Bp = (B + 127) & ~127;
    dim3 tb(32, 8);
    k_mse_grad<<<1, 1024, 0, m->stream>>>(m->Y, m->outp, m->Tf, B, m->out, m->dY, Bp, m->outp, m->G + m->g_b3, m->loss);
    RQ_CUDA(cudaGetLastError());
    // dW3^T [h2 x outp] = H2^T [h2 x Bp] * (dY^T [outp x Bp])^T
    k_transpose_bf16<<<dim3((m->h2 + 31) / 32, (Bp + 31) / 32), tb, 0, m->stream>>>(m->H2, Bp, m->h2, m->h2, m->H2t, Bp);
    k_transpose_bf16<<<dim3((m->outp + 31) / 32, (Bp + 31) / 32), tb, 0, m->stream>>>(m->dY, Bp, m->outp, m->outp, m->dYt, Bp);
    RQ_TRY(rq::gemm_bf16(m->stream, m->H2t, Bp, m->dYt, Bp, m->h2, m->outp, Bp, m->G + m->g_w3t, m->outp, EPI_F32,
                         nullptr, nullptr, 0));
    // dH2 [Bp x h2] = dY [Bp x outp] * (W3^T [h2 x outp])^T
    RQ_TRY(rq::gemm_bf16(m->stream, m->dY, m->outp, m->W3t, m->outp, Bp, m->h2, m->outp, m->dH2, m->h2, EPI_F32,
                         nullptr, nullptr, 0));
    k_relu_back<<<(m->h2 + 127) / 128, 128, 0, m->stream>>>(m->dH2, m->Z2, B, Bp, m->h2, m->dZ2, m->G + m->g_b2);
    // dW2 [h2 x h1] = dZ2^T [h2 x Bp] * (H1^T [h1 x Bp])^T
    k_transpose_bf16<<<dim3((m->h2 + 31) / 32, (Bp + 31) / 32), tb, 0, m->stream>>>(m->dZ2, Bp, m->h2, m->h2, m->dZ2t, Bp);
    k_transpose_bf16<<<dim3((m->h1 + 31) / 32, (Bp + 31) / 32), tb, 0, m->stream>>>(m->H1, Bp, m->h1, m->h1, m->H1t, Bp);
    RQ_TRY(rq::gemm_bf16(m->stream, m->dZ2t, Bp, m->H1t, Bp, m->h2, m->h1, Bp, m->G + m->g_w2, m->h1, EPI_F32, nullptr,
                         nullptr, 0));
    // dH1 [Bp x h1] = dZ2 [Bp x h2] * (W2^T [h1 x h2])^T
    RQ_TRY(rq::gemm_bf16(m->stream, m->dZ2, m->h2, m->W2t, m->h2, Bp, m->h1, m->h2, m->dH1, m->h1, EPI_F32, nullptr,
                         nullptr, 0));
    k_relu_back<<<(m->h1 + 127) / 128, 128, 0, m->stream>>>(m->dH1, m->Z1, B, Bp, m->h1, m->dZ1, m->G + m->g_b1);
    // dW1 [h1 x inp] = dZ1^T [h1 x Bp] * (X^T [inp x Bp])^T
    k_transpose_bf16<<<dim3((m->h1 + 31) / 32, (Bp + 31) / 32), tb, 0, m->stream>>>(m->dZ1, Bp, m->h1, m->h1, m->dZ1t, Bp);
    k_transpose_bf16<<<dim3((m->inp + 31) / 32, (Bp + 31) / 32), tb, 0, m->stream>>>(m->X, Bp, m->inp, m->inp, m->Xt, Bp);
    RQ_TRY(rq::gemm_bf16(m->stream, m->dZ1t, Bp, m->Xt, Bp, m->h1, m->inp, Bp, m->G + m->g_w1, m->inp, EPI_F32, nullptr,
                         nullptr, 0));
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

// one Adam step over every parameter block from m->G
int mlp_adam(rq_mlp* m, float lr, float b1, float b2, float eps) {
    m->step += 1;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    const int sms = rq::num_sms(m->device);
    struct Blk { long off, goff; int rows, cols; long gsr, gsc; };
    const Blk blks[] = {
        {m->off_w1, m->g_w1, m->h1, m->in, m->inp, 1},
        {m->off_b1, m->g_b1, 1, m->h1, 0, 1},
        {m->off_w2, m->g_w2, m->h2, m->h1, m->h1, 1},
        {m->off_b2, m->g_b2, 1, m->h2, 0, 1},
        {m->off_w3, m->g_w3t, m->out, m->h2, 1, m->outp},   // dW3 is stored transposed
        {m->off_b3, m->g_b3, 1, m->out, 0, 1},
    };
    for (const auto& b : blks) {
        k_adam<<<rq::grid_for((uint64_t)b.rows * b.cols, 256, sms), 256, 0, m->stream>>>(
            m->P + b.off, m->Mo + b.off, m->Vo + b.off, m->G + b.goff, b.rows, b.cols, b.gsr, b.gsc, lr, b1, b2, eps, c1,
            c2);
    }
    RQ_CUDA(cudaGetLastError());
    return mlp_refresh_bf16(m);
}

}  // namespace

extern "C" {

int rq_mlp_create(int32_t in, int32_t h1, int32_t h2, int32_t out, uint64_t seed, rq_mlp** res) {
    if (!res) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    if (in < 1 || h1 < 16 || h2 < 16 || out < 1 || h1 % 16 || h2 % 16)
        return rq::fail(RQ_ERR_INVALID_ARGUMENT, "mlp: hidden widths must be positive multiples of 16");
    std::unique_ptr<rq_mlp> m(new rq_mlp());
    cudaGetDevice(&m->device);
    m->in = in; m->h1 = h1; m->h2 = h2; m->out = out;
    m->inp = pad16(in);
    m->outp = (out + 31) & ~31;
    m->off_w1 = 0;
    m->off_b1 = m->off_w1 + (long)h1 * in;
    m->off_w2 = m->off_b1 + h1;
    m->off_b2 = m->off_w2 + (long)h2 * h1;
    m->off_w3 = m->off_b2 + h2;
    m->off_b3 = m->off_w3 + (long)out * h2;
    m->nparam = m->off_b3 + out;
    m->g_w1 = 0;
    m->g_b1 = m->g_w1 + (long)h1 * m->inp;
    m->g_w2 = m->g_b1 + h1;
    m->g_b2 = m->g_w2 + (long)h2 * h1;
    m->g_w3t = m->g_b2 + h2;
    m->g_b3 = m->g_w3t + (long)h2 * m->outp;
    m->g_total = m->g_b3 + m->outp;
    RQ_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    RQ_TRY(dalloc(&m->P, m->nparam));
    RQ_TRY(dalloc(&m->Mo, m->nparam));
    RQ_TRY(dalloc(&m->Vo, m->nparam));
    RQ_TRY(dalloc(&m->G, m->g_total));
    RQ_TRY(dalloc(&m->loss, 1));
    RQ_TRY(dalloc(&m->W1b, (size_t)h1 * m->inp));
    RQ_TRY(dalloc(&m->W2b, (size_t)h2 * h1));
    RQ_TRY(dalloc(&m->W3b, (size_t)m->outp * h2));
    RQ_TRY(dalloc(&m->W2t, (size_t)h1 * h2));
    RQ_TRY(dalloc(&m->W3t, (size_t)h2 * m->outp));
    RQ_CUDA(cudaMemset(m->G, 0, m->g_total * sizeof(float)));
    RQ_CUDA(cudaMemset(m->Mo, 0, m->nparam * sizeof(float)));
    RQ_CUDA(cudaMemset(m->Vo, 0, m->nparam * sizeof(float)));
    // He-uniform weights from the documented Philox stream (stream 6), zero biases
    std::vector<float> P(m->nparam, 0.f);
    uint64_t draw = 0;
    auto fill = [&](long off, int rows, int cols) {
        const double lim = std::sqrt(6.0 / cols);
        for (long k = 0; k < (long)rows * cols; ++k) P[off + k] = (float)((2.0 * rqd::uniform(seed, 6, draw++) - 1.0) * lim);
    };
    fill(m->off_w1, h1, in);
    fill(m->off_w2, h2, h1);
    fill(m->off_w3, out, h2);
    // stream-ordered: the refresh below runs on the network's (non-blocking) stream
    RQ_CUDA(cudaMemcpyAsync(m->P, P.data(), m->nparam * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    RQ_TRY(mlp_refresh_bf16(m.get()));
    RQ_CUDA(cudaStreamSynchronize(m->stream));
    *res = m.release();
    return RQ_OK;
}

int rq_mlp_destroy(rq_mlp* m) {
    if (!m) return RQ_OK;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    void* bufs[] = {m->P, m->Mo, m->Vo, m->G, m->loss, m->W1b, m->W2b, m->W3b, m->W2t, m->W3t, m->X, m->Xt, m->H1,
                    m->H1t, m->H2, m->H2t, m->dY, m->dYt, m->dZ2, m->dZ2t, m->dZ1, m->dZ1t, m->Xf, m->Tf, m->Z1,
                    m->Z2, m->Y, m->dH2, m->dH1};
    for (void* b : bufs) if (b) cudaFree(b);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return RQ_OK;
}

int rq_mlp_num_params(const rq_mlp* m, int64_t* n) {
    if (!m || !n) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    *n = m->nparam;
    return RQ_OK;
}

int rq_mlp_get_params(rq_mlp* m, float* params) {
    if (!m || !params) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_CUDA(cudaSetDevice(m->device));
    RQ_CUDA(cudaMemcpyAsync(params, m->P, m->nparam * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    RQ_CUDA(cudaStreamSynchronize(m->stream));
    return RQ_OK;
}

int rq_mlp_set_params(rq_mlp* m, const float* params) {
    if (!m || !params) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "null pointer");
    RQ_CUDA(cudaSetDevice(m->device));
    RQ_CUDA(cudaMemcpyAsync(m->P, params, m->nparam * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    RQ_CUDA(cudaMemsetAsync(m->Mo, 0, m->nparam * sizeof(float), m->stream));
    RQ_CUDA(cudaMemsetAsync(m->Vo, 0, m->nparam * sizeof(float), m->stream));
    m->step = 0;
    RQ_TRY(mlp_refresh_bf16(m));
    RQ_CUDA(cudaStreamSynchronize(m->stream));
    return RQ_OK;
}

int rq_mlp_forward(rq_mlp* m, const float* x, int32_t B, float* y) {
    if (!m || !x || !y || B < 1) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "bad argument");
    RQ_CUDA(cudaSetDevice(m->device));
    RQ_TRY(mlp_reserve(m, B));
    RQ_CUDA(cudaMemcpyAsync(m->Xf, x, (size_t)B * m->in * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    RQ_TRY(mlp_forward_dev(m, B));
    RQ_CUDA(cudaMemcpy2DAsync(y, m->out * sizeof(float), m->Y, m->outp * sizeof(float), m->out * sizeof(float), B,
                              cudaMemcpyDeviceToHost, m->stream));
    RQ_CUDA(cudaStreamSynchronize(m->stream));
    int to = 0;
    RQ_TRY(rq::mma_timeout_flag(&to));
    if (to) return rq::fail(RQ_ERR_TIMEOUT, "tensor-core wait expired");
    return RQ_OK;
}

// loss and flat gradients (same layout as the parameters) for x (B x in), targets (B x out)
int rq_mlp_gradients(rq_mlp* m, const float* x, const float* t, int32_t B, float* loss, float* grads) {
    if (!m || !x || !t || !loss || !grads || B < 1) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "bad argument");
    RQ_CUDA(cudaSetDevice(m->device));
    RQ_TRY(mlp_reserve(m, B));
    RQ_CUDA(cudaMemcpyAsync(m->Xf, x, (size_t)B * m->in * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    RQ_CUDA(cudaMemcpyAsync(m->Tf, t, (size_t)B * m->out * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    RQ_TRY(mlp_forward_dev(m, B));
    RQ_TRY(mlp_backward_dev(m, B));
    float* dflat = nullptr;
    RQ_TRY(dalloc(&dflat, m->nparam));
    const int sms = rq::num_sms(m->device);
    struct Blk { long off, goff; int rows, cols; long gsr, gsc; };
    const Blk blks[] = {
        {m->off_w1, m->g_w1, m->h1, m->in, m->inp, 1},  {m->off_b1, m->g_b1, 1, m->h1, 0, 1},
        {m->off_w2, m->g_w2, m->h2, m->h1, m->h1, 1},   {m->off_b2, m->g_b2, 1, m->h2, 0, 1},
        {m->off_w3, m->g_w3t, m->out, m->h2, 1, m->outp}, {m->off_b3, m->g_b3, 1, m->out, 0, 1},
    };
    for (const auto& b : blks)
        k_gather<<<rq::grid_for((uint64_t)b.rows * b.cols, 256, sms), 256, 0, m->stream>>>(m->G + b.goff, b.rows, b.cols,
                                                                                         b.gsr, b.gsc, dflat + b.off);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(grads, dflat, m->nparam * sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    cudaFree(dflat);
    RQ_CUDA(e);
    int to = 0;
    RQ_TRY(rq::mma_timeout_flag(&to));
    if (to) return rq::fail(RQ_ERR_TIMEOUT, "tensor-core wait expired");
    return RQ_OK;
}

// `steps` Adam steps over minibatches x (n x in), t (n x out): minibatch k uses rows
// [k*B mod n ...) wrapping; returns the mean loss of the last step
int rq_mlp_train(rq_mlp* m, const float* x, const float* t, int32_t n, int32_t B, int32_t steps, float lr,
                 float* last_loss) {
    if (!m || !x || !t || n < 1 || B < 1 || steps < 0) return rq::fail(RQ_ERR_INVALID_ARGUMENT, "bad argument");
    RQ_CUDA(cudaSetDevice(m->device));
    RQ_TRY(mlp_reserve(m, B));
    float *dx = nullptr, *dt = nullptr;
    RQ_TRY(dalloc(&dx, (size_t)n * m->in));
    RQ_TRY(dalloc(&dt, (size_t)n * m->out));
    int rc = RQ_OK;
    cudaError_t e = cudaMemcpyAsync(dx, x, (size_t)n * m->in * sizeof(float), cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, t, (size_t)n * m->out * sizeof(float), cudaMemcpyHostToDevice, m->stream);
    if (e != cudaSuccess) rc = rq::cuda_fail(e, "cudaMemcpyAsync");
    for (int s = 0; s < steps && rc == RQ_OK; ++s) {
        const long r0 = ((long)s * B) % n;
        const int take = (int)std::min<long>(B, n - r0);
        e = cudaMemcpyAsync(m->Xf, dx + r0 * m->in, (size_t)take * m->in * sizeof(float), cudaMemcpyDeviceToDevice, m->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(m->Tf, dt + r0 * m->out, (size_t)take * m->out * sizeof(float), cudaMemcpyDeviceToDevice,
                                m->stream);
        if (e != cudaSuccess) { rc = rq::cuda_fail(e, "cudaMemcpyAsync"); break; }
        rc = mlp_forward_dev(m, take);
        if (rc == RQ_OK) rc = mlp_backward_dev(m, take);
        if (rc == RQ_OK) rc = mlp_adam(m, lr, 0.9f, 0.999f, 1e-8f);
    }
    if (rc == RQ_OK && last_loss) {
        e = cudaMemcpyAsync(last_loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
        if (e != cudaSuccess) rc = rq::cuda_fail(e, "cudaMemcpyAsync");
    }
    e = cudaStreamSynchronize(m->stream);
    cudaFree(dx);
    cudaFree(dt);
    RQ_TRY(rc);
    RQ_CUDA(e);
    int to = 0;
    RQ_TRY(rq::mma_timeout_flag(&to));
    if (to) return rq::fail(RQ_ERR_TIMEOUT, "tensor-core wait expired");
    return RQ_OK;
}

}  // extern "C"
