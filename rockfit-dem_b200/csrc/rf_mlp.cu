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
