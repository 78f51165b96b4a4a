// BF16 tensor-core GEMM for sm_100a (tcgen05 + TMEM) and the warm-start MLP built on it.
//
// rf_gemm_bf16 computes C[M x N] = A[M x K] * B[N x K]^T with both operands K-major
// (row-major with K contiguous), BF16 inputs and FP32 accumulation in tensor memory:
//   - one CTA of 128 threads per 128-row tile of C (grid.x), the whole N (<= 256) per
//     CTA, K split over grid.y (split-K results are added atomically);
//   - K is walked in chunks of 64: the four warps stage the A chunk (128 x 64) and the
//     B chunk (N x 64) in shared memory in the canonical no-swizzle K-major layout
//     (8-row x 16-byte core matrices; 128 bytes between K-adjacent core matrices,
//     1024 bytes between 8-row groups), one elected thread issues four
//     tcgen05.mma.kind::f16 (M=128, K=16 each) into the TMEM accumulator and commits
//     them to an mbarrier that all threads wait on (bounded);
//   - the epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes
//     32w..32w+31, one row per thread) and applies bias/ReLU, the ReLU mask of the
//     backward pass, or the split-K atomic add, writing BF16 rows, their transpose
//     (the next GEMM's K-major operand) or FP32.
// Waits give up after a bounded number of polls, raise an error flag and still free the
// tensor memory before returning.
#include <cuda_bf16.h>
#include <cstring>
#include <cmath>
#include <vector>
#include "rf_common.cuh"

namespace rf {
namespace mlp {

enum Epi : int {
    EPI_RELU_BF16 = 0,      // h = relu(acc + bias) -> bf16 rows (+ transpose)
    EPI_LINEAR_F32 = 1,     // y = acc + bias -> fp32, first ncols_f columns
    EPI_MASK_BF16 = 2,      // dz = acc * (mask > 0) -> bf16 rows (+ transpose)
    EPI_ATOMIC_F32 = 3,     // out += scale * acc (split-K weight gradients)
};

struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    int M, N, K, lda, ldb;
    int chunks_per_split;
    int mode;
    const float* bias;
    const __nv_bfloat16* mask;
    int ldm;
    __nv_bfloat16* out_h;
    int ld_h;
    __nv_bfloat16* out_ht;
    int ld_ht;
    float* out_f;
    int ld_f, ncols_f;
    float scale;
    uint32_t* err;
};

#define GEMM_KC 64                      // K per staged chunk (four MMAs of K = 16)
#define GEMM_A_BYTES (128 * GEMM_KC * 2)
#define GEMM_B_MAX_BYTES (256 * GEMM_KC * 2)
#define GEMM_WAIT_LIMIT (1u << 24)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: canonical K-major layout without swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);            // start address
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;        // leading byte offset: K-adjacent core matrices
    d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;       // stride byte offset: 8-row groups
    d |= (uint64_t)1 << 46;                              // descriptor version (sm_100)
    return d;                                            // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: D = F32, A = B = BF16, both K-major, M = 128.
__host__ __device__ __forceinline__ uint32_t umma_idesc(int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (uint32_t it = 0; it < GEMM_WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Copy the 16-byte pieces of a rows x 64 chunk (rows from r0, columns from k0) into the
// canonical layout; rows >= nrows and columns >= K read as zero.
__device__ __forceinline__ void stage_chunk(uint8_t* s, const __nv_bfloat16* g, int ld, int r0, int nrows, int rows,
                                            int k0, int K) {
    const int pieces = rows * (GEMM_KC / 8);
    for (int p = threadIdx.x; p < pieces; p += blockDim.x) {
        const int r = p >> 3, kg = p & 7;
        const int gr = r0 + r, gk = k0 + kg * 8;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (gr < nrows && gk < K) v = *reinterpret_cast<const uint4*>(g + (size_t)gr * ld + gk);
        *reinterpret_cast<uint4*>(s + (r >> 3) * 1024 + kg * 128 + (r & 7) * 16) = v;
    }
}

template <int NC>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[NC]);
template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

__global__ void __launch_bounds__(128) k_umma_gemm(GemmArgs g) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sA = smem;
    uint8_t* sB = smem + GEMM_A_BYTES;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_taddr;
    __shared__ uint32_t s_fail;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * 128;
    const int ncols = g.N <= 32 ? 32 : (g.N <= 64 ? 64 : (g.N <= 128 ? 128 : 256));
    const uint32_t bar_a = smem_u32(&bar);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_taddr)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t taddr = s_taddr;
    const int nchunks = (g.K + GEMM_KC - 1) / GEMM_KC;
    const int c0 = blockIdx.y * g.chunks_per_split;
    const int c1 = min(nchunks, c0 + g.chunks_per_split);
    const uint32_t idesc = umma_idesc(g.N);
    uint32_t phase = 0;
    bool ok = true;
    for (int c = c0; c < c1 && ok; ++c) {
        stage_chunk(sA, g.A, g.lda, m0, g.M, 128, c * GEMM_KC, g.K);
        stage_chunk(sB, g.B, g.ldb, 0, g.N, g.N, c * GEMM_KC, g.K);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // generic writes -> tensor core reads
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
            for (int s = 0; s < GEMM_KC / 16; ++s) {
                const uint64_t da = umma_desc(smem_u32(sA + s * 256));
                const uint64_t db = umma_desc(smem_u32(sB + s * 256));
                const uint32_t acc = (c > c0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    :
                    : "r"(taddr), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar_a)
                         : "memory");
        }
        if (!mbar_wait(bar_a, phase)) {
            atomicOr(&s_fail, 1u);
        }
        phase ^= 1u;
        __syncthreads();                                 // the staging buffers are free again
        ok = (s_fail == 0);
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    }
    if (!ok) {
        if (threadIdx.x == 0 && g.err) atomicOr(g.err, 1u);
    } else if (c1 > c0) {
        // epilogue: thread (warp w, lane l) owns row m0 + 32w + l
        const int row = m0 + warp * 32 + lane;
        for (int cb = 0; cb < g.N; cb += 16) {
            float v[16];
            tmem_ld<16>(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, v);
            if (row >= g.M) continue;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int col = cb + q;
                if (col >= g.N) break;
                float a = v[q];
                switch (g.mode) {
                    case EPI_RELU_BF16: {
                        a = fmaxf(a + (g.bias ? g.bias[col] : 0.f), 0.f);
                        const __nv_bfloat16 h = __float2bfloat16_rn(a);
                        g.out_h[(size_t)row * g.ld_h + col] = h;
                        if (g.out_ht) g.out_ht[(size_t)col * g.ld_ht + row] = h;
                        break;
                    }
                    case EPI_LINEAR_F32:
                        if (col < g.ncols_f) g.out_f[(size_t)row * g.ld_f + col] = (a + (g.bias ? g.bias[col] : 0.f)) * g.scale;
                        break;
                    case EPI_MASK_BF16: {
                        const float m = __bfloat162float(g.mask[(size_t)row * g.ldm + col]);
                        const __nv_bfloat16 h = __float2bfloat16_rn(m > 0.f ? a : 0.f);
                        g.out_h[(size_t)row * g.ld_h + col] = h;
                        if (g.out_ht) g.out_ht[(size_t)col * g.ld_ht + row] = h;
                        break;
                    }
                    default:
                        if (col < g.ncols_f) atomicAdd(&g.out_f[(size_t)row * g.ld_f + col], g.scale * a);
                        break;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
    }
}

}  // namespace mlp
}  // namespace rf

using namespace rf;
using namespace rf::mlp;

namespace {
uint32_t* gemm_err_word() {
    static thread_local uint32_t* w = nullptr;
    if (!w) {
        if (cudaMalloc(&w, sizeof(uint32_t)) != cudaSuccess) return nullptr;
        cudaMemset(w, 0, sizeof(uint32_t));
    }
    return w;
}
}  // namespace

extern "C" rf_status rf_gemm_bf16(const void* A, int lda, const void* B, int ldb, int M, int N, int K, int mode,
                                  const float* bias, const void* mask, int ldm, void* out_h, int ld_h, void* out_ht,
                                  int ld_ht, float* out_f, int ld_f, int ncols_f, float scale, int splits,
                                  rf_stream stream) {
    if (!A || !B || M <= 0 || N <= 0 || K <= 0 || N > 256 || (N % 16) != 0 || (K % 8) != 0 || (lda % 8) != 0 ||
        (ldb % 8) != 0 || lda < K || ldb < K || mode < 0 || mode > 3 || splits <= 0 ||
        ((uintptr_t)A % 16) != 0 || ((uintptr_t)B % 16) != 0) {
        set_error("rf_gemm_bf16: bad arguments (N multiple of 16 up to 256, K and leading dims multiples of 8, "
                  "16-byte aligned operands)");
        return RF_ERR_INVALID;
    }
    if ((mode == EPI_RELU_BF16 || mode == EPI_MASK_BF16) && (!out_h || ld_h < N || (mode == EPI_MASK_BF16 && !mask))) {
        set_error("rf_gemm_bf16: bf16 epilogue needs out_h (and mask)");
        return RF_ERR_INVALID;
    }
    if ((mode == EPI_LINEAR_F32 || mode == EPI_ATOMIC_F32) && (!out_f || ncols_f <= 0 || ncols_f > N)) {
        set_error("rf_gemm_bf16: fp32 epilogue needs out_f and 0 < ncols_f <= N");
        return RF_ERR_INVALID;
    }
    if (mode != EPI_ATOMIC_F32 && splits != 1) {
        set_error("rf_gemm_bf16: split-K only with the atomic epilogue");
        return RF_ERR_INVALID;
    }
    uint32_t* err = gemm_err_word();
    if (!err) { set_error("rf_gemm_bf16: no status word"); return RF_ERR_CUDA; }
    GemmArgs g;
    std::memset(&g, 0, sizeof(g));
    g.A = (const __nv_bfloat16*)A; g.B = (const __nv_bfloat16*)B;
    g.M = M; g.N = N; g.K = K; g.lda = lda; g.ldb = ldb;
    const int nchunks = (K + GEMM_KC - 1) / GEMM_KC;
    const int sp = splits > nchunks ? nchunks : splits;
    g.chunks_per_split = (nchunks + sp - 1) / sp;
    g.mode = mode; g.bias = bias; g.mask = (const __nv_bfloat16*)mask; g.ldm = ldm;
    g.out_h = (__nv_bfloat16*)out_h; g.ld_h = ld_h; g.out_ht = (__nv_bfloat16*)out_ht; g.ld_ht = ld_ht;
    g.out_f = out_f; g.ld_f = ld_f; g.ncols_f = ncols_f; g.scale = scale; g.err = err;
    const size_t smem = GEMM_A_BYTES + (size_t)N * GEMM_KC * 2;
    static bool attr_set = false;
    if (!attr_set) {
        RF_CUDA(cudaFuncSetAttribute(k_umma_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     GEMM_A_BYTES + GEMM_B_MAX_BYTES));
        attr_set = true;
    }
    const int gy = (nchunks + g.chunks_per_split - 1) / g.chunks_per_split;
    dim3 grid((M + 127) / 128, gy);
    k_umma_gemm<<<grid, 128, smem, (cudaStream_t)stream>>>(g);
    RF_CHECK_LAUNCH("k_umma_gemm");
    return RF_OK;
}

// Read and clear the GEMM status word (1 = an MMA completion wait gave up).
extern "C" rf_status rf_gemm_status(rf_stream stream) {
    uint32_t* err = gemm_err_word();
    if (!err) return RF_ERR_CUDA;
    uint32_t h = 0;
    RF_CUDA(cudaMemcpyAsync(&h, err, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    RF_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (h) {
        RF_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), (cudaStream_t)stream));
        set_error("rf_gemm_bf16: tensor-core completion wait timed out");
        return RF_ERR_CUDA;
    }
    return RF_OK;
}

// ===========================================================================
// Warm-start MLP: 64 -> 128 -> 128 -> 128 -> 6 (padded to 16), ReLU, BF16 weights and
// activations, FP32 accumulation (rf_gemm_bf16), FP32 master weights trained with Adam
// on the mean squared error. Weights are kept in the layout of a linear layer,
// W[out][in], which is the K-major B operand of the forward GEMMs; a BF16 transpose
// W^T[in][out] is the B operand of the backward GEMMs dH = dZ W. Weight gradients come
// out of the GEMM as dW^T[in][out] = H^T dZ (K = the particles, split-K).
// ===========================================================================
namespace rf {
namespace mlp {

static const int NL = 4;
static const int DIN[NL] = {64, 128, 128, 128};
static const int DOUT[NL] = {128, 128, 128, 16};     // the last layer's 6 outputs padded to 16
static const int NOUT = 6;

__global__ void k_init_weights(float* W, float* b, int out, int in, int out_real, uint64_t seed) {
    const int n = out * in;
    const float bound = sqrtf(6.0f / (float)in) * (out_real < out ? 0.1f : 1.0f);   // He-uniform; small last layer
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int o = q / in;
        uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(q + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const float u = (float)(z >> 40) * (1.0f / 16777216.0f);
        W[q] = o < out_real ? (2.0f * u - 1.0f) * bound : 0.f;
    }
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < out; q += gridDim.x * blockDim.x) b[q] = 0.f;
}

// BF16 copies of W[out][in] in both layouts.
__global__ void k_weights_bf16(const float* W, int out, int in, __nv_bfloat16* Wb, __nv_bfloat16* WbT) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < out * in; q += gridDim.x * blockDim.x) {
        const int o = q / in, i = q - o * in;
        const __nv_bfloat16 h = __float2bfloat16_rn(W[q]);
        Wb[q] = h;
        WbT[(size_t)i * out + o] = h;
    }
}

// Output gradient of the loss mean((y - t)^2) over the rows and the NOUT outputs:
// fp32 for the bias gradient, bf16 rows and transpose for the GEMMs; the per-block
// partial loss in double.
__global__ void k_out_grad(const float* Y, const float* T, int rows, int rows_pad, float* dY, __nv_bfloat16* dZ,
                           __nv_bfloat16* dZT, double* loss_part) {
    const float inv = 2.0f / ((float)rows * (float)NOUT);
    double l = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows_pad; r += gridDim.x * blockDim.x) {
        for (int c = 0; c < 16; ++c) {
            float g = 0.f;
            if (r < rows && c < NOUT) {
                const float e = Y[(size_t)r * 16 + c] - T[(size_t)r * NOUT + c];
                l += (double)e * e;
                g = inv * e;
            }
            dY[(size_t)r * 16 + c] = g;
            const __nv_bfloat16 h = __float2bfloat16_rn(g);
            dZ[(size_t)r * 16 + c] = h;
            dZT[(size_t)c * rows_pad + r] = h;
        }
    }
    __shared__ double sh[8];
    for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
        loss_part[blockIdx.x] = s;
    }
}

// Bias gradient: column sums of a [rows x n] gradient (fp32 or bf16), one block per column.
template <class T>
__global__ void k_colsum(const T* G, int rows, int ld, float* out) {
    const int c = blockIdx.x;
    float s = 0.f;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) s += (float)G[(size_t)r * ld + c];
    __shared__ float sh[8];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        out[c] = t;
    }
}

// Residual mode: y[r][c] += sign * x[r][c] for the first NOUT columns (x bf16 [rows][64]).
__global__ void k_add_input(float* Y, int ldy, int ncols, const __nv_bfloat16* X, int rows, float sign) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rows * NOUT; q += gridDim.x * blockDim.x) {
        const int r = q / NOUT, c = q - r * NOUT;
        if (c < ncols) Y[(size_t)r * ldy + c] += sign * __bfloat162float(X[(size_t)r * 64 + c]);
    }
}

// dst[c][r] = src[r][c] for a [rows x cols] bf16 matrix (32 x 32 tiles through shared memory).
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ src, int rows, int cols,
                                 __nv_bfloat16* __restrict__ dst, int ldd) {
    __shared__ __nv_bfloat16 t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        t[y][threadIdx.x] = (r < rows && c < cols) ? src[(size_t)r * cols + c] : __float2bfloat16_rn(0.f);
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        if (c < cols && r < rows) dst[(size_t)c * ldd + r] = t[threadIdx.x][y];
    }
}

// Adam on W[out][in] with gradient gT[in][out] (and the bias), then the bf16 copies.
__global__ void k_adam(float* W, float* mW, float* vW, const float* gT, float* b, float* mb, float* vb, const float* gb,
                       int out, int in, int out_real, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* Wb, __nv_bfloat16* WbT) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < out * in; q += gridDim.x * blockDim.x) {
        const int o = q / in, i = q - o * in;
        if (o >= out_real) continue;
        const float g = gT[(size_t)i * out + o];
        const float m = b1 * mW[q] + (1.f - b1) * g, v = b2 * vW[q] + (1.f - b2) * g * g;
        mW[q] = m; vW[q] = v;
        W[q] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
        const __nv_bfloat16 h = __float2bfloat16_rn(W[q]);
        Wb[q] = h;
        WbT[(size_t)i * out + o] = h;
    }
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < out_real; o += gridDim.x * blockDim.x) {
        const float g = gb[o];
        const float m = b1 * mb[o] + (1.f - b1) * g, v = b2 * vb[o] + (1.f - b2) * g * g;
        mb[o] = m; vb[o] = v;
        b[o] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    }
}

}  // namespace mlp
}  // namespace rf

struct rf_mlp {
    int rows_cap = 0;           // activation capacity (rows, multiple of 128)
    float *W[rf::mlp::NL] = {}, *b[rf::mlp::NL] = {};
    float *mW[rf::mlp::NL] = {}, *vW[rf::mlp::NL] = {}, *mb[rf::mlp::NL] = {}, *vb[rf::mlp::NL] = {};
    float *gT[rf::mlp::NL] = {}, *gb[rf::mlp::NL] = {};
    __nv_bfloat16 *Wb[rf::mlp::NL] = {}, *WbT[rf::mlp::NL] = {};
    __nv_bfloat16 *H[rf::mlp::NL] = {}, *HT[rf::mlp::NL] = {};    // H[0] = input features
    __nv_bfloat16 *dZ[rf::mlp::NL] = {}, *dZT[rf::mlp::NL] = {};  // gradient at each layer's output
    float *Y = nullptr, *dY = nullptr, *Tres = nullptr;
    double* loss_part = nullptr;
    int steps = 0;
    int residual = 0;           // predict the correction to the input's first 6 features
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
};

namespace {
using namespace rf::mlp;

template <class T> rf_status mlp_alloc(rf_mlp* m, T** p, size_t n) {
    void* q = nullptr;
    RF_CUDA(cudaMalloc(&q, (n ? n : 1) * sizeof(T)));
    m->allocs.push_back(q);
    *p = (T*)q;
    return RF_OK;
}

rf_status mlp_reserve(rf_mlp* m, int rows) {
    const int need = (rows + 127) / 128 * 128;
    if (need <= m->rows_cap) return RF_OK;
    for (int l = 0; l < NL; ++l) {
        if (m->H[l]) { cudaFree(m->H[l]); cudaFree(m->HT[l]); cudaFree(m->dZ[l]); cudaFree(m->dZT[l]); }
    }
    if (m->Y) { cudaFree(m->Y); cudaFree(m->dY); cudaFree(m->loss_part); cudaFree(m->Tres); }
    for (int l = 0; l < NL; ++l) {
        RF_CUDA(cudaMalloc(&m->H[l], (size_t)need * DIN[l] * 2));
        RF_CUDA(cudaMalloc(&m->HT[l], (size_t)need * DIN[l] * 2));
        RF_CUDA(cudaMalloc(&m->dZ[l], (size_t)need * DOUT[l] * 2));
        RF_CUDA(cudaMalloc(&m->dZT[l], (size_t)need * DOUT[l] * 2));
    }
    RF_CUDA(cudaMalloc(&m->Y, (size_t)need * 16 * sizeof(float)));
    RF_CUDA(cudaMalloc(&m->dY, (size_t)need * 16 * sizeof(float)));
    RF_CUDA(cudaMalloc(&m->loss_part, 1024 * sizeof(double)));
    RF_CUDA(cudaMalloc(&m->Tres, (size_t)need * NOUT * sizeof(float)));
    // zero everything once: the padding rows past a call's row count are never written by
    // the forward pass, but the weight gradients sum over them (with zero output gradients),
    // and 0 * NaN from uninitialised memory would poison the sums
    for (int l = 0; l < NL; ++l) {
        RF_CUDA(cudaMemsetAsync(m->H[l], 0, (size_t)need * DIN[l] * 2, m->stream));
        RF_CUDA(cudaMemsetAsync(m->HT[l], 0, (size_t)need * DIN[l] * 2, m->stream));
        RF_CUDA(cudaMemsetAsync(m->dZ[l], 0, (size_t)need * DOUT[l] * 2, m->stream));
        RF_CUDA(cudaMemsetAsync(m->dZT[l], 0, (size_t)need * DOUT[l] * 2, m->stream));
    }
    RF_CUDA(cudaMemsetAsync(m->Y, 0, (size_t)need * 16 * sizeof(float), m->stream));
    RF_CUDA(cudaMemsetAsync(m->dY, 0, (size_t)need * 16 * sizeof(float), m->stream));
    m->rows_cap = need;
    return RF_OK;
}

// Forward over `rows` feature rows X (bf16 [rows x 64], ld 64). With `keep`, the hidden
// activations and their transposes stay for the backward pass. Y: fp32 [rows x 16].
rf_status mlp_forward(rf_mlp* m, const __nv_bfloat16* X, int rows, bool keep, float* Yout, int ldy, int ncols) {
    const int rp = (rows + 127) / 128 * 128;
    rf_stream s = (rf_stream)m->stream;
    const void* in = X;
    for (int l = 0; l < NL - 1; ++l) {
        if (rf_status st = rf_gemm_bf16(in, DIN[l], m->Wb[l], DIN[l], rows, DOUT[l], DIN[l], EPI_RELU_BF16, m->b[l],
                                        nullptr, 0, m->H[l + 1], DOUT[l], keep ? m->HT[l + 1] : nullptr, rp, nullptr, 0,
                                        0, 1.f, 1, s))
            return st;
        in = m->H[l + 1];
    }
    return rf_gemm_bf16(in, DIN[NL - 1], m->Wb[NL - 1], DIN[NL - 1], rows, DOUT[NL - 1], DIN[NL - 1], EPI_LINEAR_F32,
                        m->b[NL - 1], nullptr, 0, nullptr, 0, nullptr, 0, Yout, ldy, ncols, 1.f, 1, s);
}
}  // namespace

extern "C" {

rf_status rf_mlp_create(uint64_t seed, rf_mlp** out) {
    if (!out) { set_error("rf_mlp_create: null output"); return RF_ERR_INVALID; }
    rf_mlp* m = new rf_mlp();
    auto fail = [&](rf_status s) { rf_mlp_destroy(m); return s; };
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(RF_ERR_CUDA);
    for (int l = 0; l < NL; ++l) {
        const size_t n = (size_t)DOUT[l] * DIN[l];
        rf_status st;
        if ((st = mlp_alloc(m, &m->W[l], n)) || (st = mlp_alloc(m, &m->b[l], DOUT[l])) ||
            (st = mlp_alloc(m, &m->mW[l], n)) || (st = mlp_alloc(m, &m->vW[l], n)) ||
            (st = mlp_alloc(m, &m->mb[l], DOUT[l])) || (st = mlp_alloc(m, &m->vb[l], DOUT[l])) ||
            (st = mlp_alloc(m, &m->gT[l], n)) || (st = mlp_alloc(m, &m->gb[l], DOUT[l])) ||
            (st = mlp_alloc(m, &m->Wb[l], n)) || (st = mlp_alloc(m, &m->WbT[l], n)))
            return fail(st);
        cudaMemsetAsync(m->mW[l], 0, n * 4, m->stream);
        cudaMemsetAsync(m->vW[l], 0, n * 4, m->stream);
        cudaMemsetAsync(m->mb[l], 0, DOUT[l] * 4, m->stream);
        cudaMemsetAsync(m->vb[l], 0, DOUT[l] * 4, m->stream);
        k_init_weights<<<64, 256, 0, m->stream>>>(m->W[l], m->b[l], DOUT[l], DIN[l], l == NL - 1 ? NOUT : DOUT[l],
                                                   seed + 1000003ull * l);
        k_weights_bf16<<<64, 256, 0, m->stream>>>(m->W[l], DOUT[l], DIN[l], m->Wb[l], m->WbT[l]);
    }
    if (cudaStreamSynchronize(m->stream) != cudaSuccess) return fail(cuda_status(cudaGetLastError(), "rf_mlp_create"));
    *out = m;
    return RF_OK;
}

rf_status rf_mlp_destroy(rf_mlp* m) {
    if (!m) return RF_OK;
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (void* p : m->allocs) cudaFree(p);
    for (int l = 0; l < NL; ++l) {
        if (m->H[l]) { cudaFree(m->H[l]); cudaFree(m->HT[l]); cudaFree(m->dZ[l]); cudaFree(m->dZT[l]); }
    }
    if (m->Y) { cudaFree(m->Y); cudaFree(m->dY); cudaFree(m->loss_part); cudaFree(m->Tres); }
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return RF_OK;
}

rf_stream rf_mlp_stream(rf_mlp* m) { return m ? (rf_stream)m->stream : nullptr; }

// Inference: Y[rows][ldy] (fp32, first ncols <= 16 outputs) from X (bf16 [rows][64]).
rf_status rf_mlp_forward(rf_mlp* m, const void* X, int rows, float* Y, int ldy, int ncols) {
    if (!m || !X || !Y || rows <= 0 || ncols <= 0 || ncols > 16 || ldy < ncols) {
        set_error("rf_mlp_forward: bad arguments");
        return RF_ERR_INVALID;
    }
    if (rf_status st = mlp_reserve(m, rows)) return st;
    if (rf_status st = mlp_forward(m, (const __nv_bfloat16*)X, rows, false, Y, ldy, ncols)) return st;
    if (m->residual) {
        k_add_input<<<256, 256, 0, m->stream>>>(Y, ldy, ncols, (const __nv_bfloat16*)X, rows, 1.f);
        RF_CHECK_LAUNCH("k_add_input");
    }
    return RF_OK;
}

// Residual mode on/off: the network's output is added to the input's first 6 features
// (the last increment's motion in the warm-start features), and trained on the difference.
rf_status rf_mlp_set_residual(rf_mlp* m, int on) {
    if (!m) { set_error("rf_mlp_set_residual: null"); return RF_ERR_INVALID; }
    m->residual = on ? 1 : 0;
    return RF_OK;
}

// Gradients of the loss mean((y - t)^2) for X (bf16 [rows][64]) and targets T (fp32
// [rows][6]); *loss receives the loss before the update. With lr > 0 an Adam step
// (beta 0.9, 0.999, eps 1e-8) follows.
rf_status rf_mlp_train_step(rf_mlp* m, const void* X, const float* T, int rows, float lr, double* loss) {
    if (!m || !X || !T || rows <= 0) { set_error("rf_mlp_train_step: bad arguments"); return RF_ERR_INVALID; }
    if (rf_status st = mlp_reserve(m, rows)) return st;
    const int rp = (rows + 127) / 128 * 128;
    cudaStream_t cs = m->stream;
    rf_stream s = (rf_stream)cs;
    // the input and its transpose (K-major operand of the first weight gradient)
    RF_CUDA(cudaMemcpyAsync(m->H[0], X, (size_t)rows * 64 * 2, cudaMemcpyDeviceToDevice, cs));
    if (rp > rows) RF_CUDA(cudaMemsetAsync(m->H[0] + (size_t)rows * 64, 0, (size_t)(rp - rows) * 64 * 2, cs));
    if (rf_status st = mlp_forward(m, m->H[0], rows, true, m->Y, 16, 16)) return st;
    const int nb = 512;
    if (m->residual) {            // the network learns T - x[0:6]: add x back to its output
        k_add_input<<<256, 256, 0, cs>>>(m->Y, 16, NOUT, m->H[0], rows, 1.f);
        RF_CHECK_LAUNCH("k_add_input");
    }
    k_out_grad<<<nb, 256, 0, cs>>>(m->Y, T, rows, rp, m->dY, m->dZ[NL - 1], m->dZT[NL - 1], m->loss_part);
    RF_CHECK_LAUNCH("k_out_grad");
    const int splits = std::max(1, std::min(64, rp / 2048));
    for (int l = NL - 1; l >= 0; --l) {
        const size_t n = (size_t)DOUT[l] * DIN[l];
        RF_CUDA(cudaMemsetAsync(m->gT[l], 0, n * 4, cs));
        // dW^T[in][out] = H_l^T[in][rows] * dZ_l^T[out][rows]^T
        const __nv_bfloat16* Hl_T = (l == 0) ? nullptr : m->HT[l];
        if (l == 0) {                       // the input's transpose, once per step
            k_transpose_bf16<<<dim3((rp + 31) / 32, 64 / 32), dim3(32, 8), 0, cs>>>(m->H[0], rp, 64, m->HT[0], rp);
            RF_CHECK_LAUNCH("k_transpose_bf16");
            Hl_T = m->HT[0];
        }
        if (rf_status st = rf_gemm_bf16(Hl_T, rp, m->dZT[l], rp, DIN[l], DOUT[l], rp, EPI_ATOMIC_F32, nullptr, nullptr,
                                        0, nullptr, 0, nullptr, 0, m->gT[l], DOUT[l], DOUT[l], 1.f, splits, s))
            return st;
        if (l == NL - 1) k_colsum<float><<<DOUT[l], 256, 0, cs>>>(m->dY, rp, 16, m->gb[l]);
        else k_colsum<__nv_bfloat16><<<DOUT[l], 256, 0, cs>>>(m->dZ[l], rp, DOUT[l], m->gb[l]);
        RF_CHECK_LAUNCH("k_colsum");
        if (l > 0) {
            // dZ_{l-1} = (dZ_l * W_l) masked by H_l > 0:  A = dZ_l [rows][out], B = W_l^T [in][out]
            if (rf_status st = rf_gemm_bf16(m->dZ[l], DOUT[l], m->WbT[l], DOUT[l], rp, DIN[l], DOUT[l], EPI_MASK_BF16,
                                            nullptr, m->H[l], DIN[l], m->dZ[l - 1], DIN[l], m->dZT[l - 1], rp, nullptr,
                                            0, 0, 1.f, 1, s))
                return st;
        }
    }
    std::vector<double> lp(nb);
    RF_CUDA(cudaMemcpyAsync(lp.data(), m->loss_part, nb * sizeof(double), cudaMemcpyDeviceToHost, cs));
    if (lr > 0.f) {
        m->steps += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)m->steps), c2 = 1.f - std::pow(b2, (float)m->steps);
        for (int l = 0; l < NL; ++l)
            k_adam<<<64, 256, 0, cs>>>(m->W[l], m->mW[l], m->vW[l], m->gT[l], m->b[l], m->mb[l], m->vb[l], m->gb[l],
                                        DOUT[l], DIN[l], l == NL - 1 ? NOUT : DOUT[l], lr, b1, b2, 1e-8f, c1, c2,
                                        m->Wb[l], m->WbT[l]);
        RF_CHECK_LAUNCH("k_adam");
    }
    RF_CUDA(cudaStreamSynchronize(cs));
    if (rf_status st = rf_gemm_status(s)) return st;
    if (loss) {
        double t = 0.0;
        for (double v : lp) t += v;
        *loss = t / ((double)rows * NOUT);
    }
    return RF_OK;
}

// Copy the fp32 weights out / in (host buffers; W[l] is [out][in] with the last layer's
// out = 16 rows, of which the first 6 are used). Layer sizes: 128x64, 128x128, 128x128, 16x128.
rf_status rf_mlp_get(rf_mlp* m, int layer, float* W, float* b) {
    if (!m || layer < 0 || layer >= NL) { set_error("rf_mlp_get: bad arguments"); return RF_ERR_INVALID; }
    RF_CUDA(cudaStreamSynchronize(m->stream));
    if (W) RF_CUDA(cudaMemcpy(W, m->W[layer], (size_t)DOUT[layer] * DIN[layer] * 4, cudaMemcpyDeviceToHost));
    if (b) RF_CUDA(cudaMemcpy(b, m->b[layer], (size_t)DOUT[layer] * 4, cudaMemcpyDeviceToHost));
    return RF_OK;
}
rf_status rf_mlp_set(rf_mlp* m, int layer, const float* W, const float* b) {
    if (!m || layer < 0 || layer >= NL || !W || !b) { set_error("rf_mlp_set: bad arguments"); return RF_ERR_INVALID; }
    RF_CUDA(cudaStreamSynchronize(m->stream));
    RF_CUDA(cudaMemcpy(m->W[layer], W, (size_t)DOUT[layer] * DIN[layer] * 4, cudaMemcpyHostToDevice));
    RF_CUDA(cudaMemcpy(m->b[layer], b, (size_t)DOUT[layer] * 4, cudaMemcpyHostToDevice));
    k_weights_bf16<<<64, 256, 0, m->stream>>>(m->W[layer], DOUT[layer], DIN[layer], m->Wb[layer], m->WbT[layer]);
    RF_CHECK_LAUNCH("k_weights_bf16");
    RF_CUDA(cudaStreamSynchronize(m->stream));
    return RF_OK;
}
// The gradients of the last rf_mlp_train_step: gT is [in][out] (the transpose of W's layout).
rf_status rf_mlp_grad(rf_mlp* m, int layer, float* gT, float* gb) {
    if (!m || layer < 0 || layer >= NL) { set_error("rf_mlp_grad: bad arguments"); return RF_ERR_INVALID; }
    RF_CUDA(cudaStreamSynchronize(m->stream));
    if (gT) RF_CUDA(cudaMemcpy(gT, m->gT[layer], (size_t)DOUT[layer] * DIN[layer] * 4, cudaMemcpyDeviceToHost));
    if (gb) RF_CUDA(cudaMemcpy(gb, m->gb[layer], (size_t)DOUT[layer] * 4, cudaMemcpyDeviceToHost));
    return RF_OK;
}

}  // extern "C"
