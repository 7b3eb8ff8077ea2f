// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05, accumulator in
// TMEM), for the learned warm-start network's layers: D (M x N, FP32, row-major) (+)=
// A (M x K) B (N x K)^T, both operands K-major BF16 (row-major with K contiguous).
//
// One CTA of 128 threads per 128 x 128 output tile and K slice (split-K over gridDim.z):
//  * operands reach shared memory by 16-byte cp.async in the canonical no-swizzle K-major
//    UMMA layout -- 8-row x 16-byte core matrices, 128 contiguous bytes each; the two core
//    matrices of one K = 16 instruction 128 bytes apart (leading byte offset), successive
//    8-row groups 1024 bytes apart (stride byte offset) -- in a 4-stage ring of 64-wide K tiles;
//  * one thread issues the four tcgen05.mma (kind::f16, M = N = 128, K = 16) of a stage and
//    commits them to the stage's mbarrier, which the ring waits on before overwriting it;
//  * the accumulator lives in 128 TMEM columns; the epilogue reads it with tcgen05.ld
//    (each warp its 32 lanes = 32 rows) and stores, or atomically adds for split-K.
// Every wait is bounded: on timeout the kernel records an error word, stops issuing, waits
// (bounded) for its own MMAs, frees its TMEM and returns.
//
// The descriptor bit layouts follow the sm100 UMMA definitions of CUTLASS/CuTe
// (cute/arch/mma_sm100_desc.hpp): shared-memory descriptor start address >> 4 in bits
// [0,14), leading byte offset >> 4 in [16,30), stride byte offset >> 4 in [32,46), version 1
// in [46,48), layout type (0 = no swizzle) in [61,64); instruction descriptor: C format F32
// (1) at bit 4, A and B format BF16 (1) at bits 7 and 10, both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "bpf_internal.cuh"
#include "tc_gemm.cuh"

namespace bpf {

namespace {

constexpr int kTM = 128, kTN = 128, kTK = 64, kStages = 4;
constexpr int kTileBytes = kTM * kTK * 2;                  // 16 KB per operand tile
constexpr int kStageBytes = 2 * kTileBytes;                // A + B
constexpr size_t kSmemBytes = (size_t)kStages * kStageBytes + 1024;   // + alignment slack

__device__ __forceinline__ unsigned su32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned c) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(c) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned parity) {
    for (long long it = 0; it < kSpinLimit; it++) {
        if (mbar_try(b, parity)) return true;
        if (it > 32) __nanosleep(20);
    }
    return false;
}

__device__ __forceinline__ uint64_t smem_desc(unsigned addr) {
    const uint64_t lbo = 128 >> 4, sbo = 1024 >> 4;
    return (uint64_t)((addr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTN >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     su32(bar))
                 : "memory");
}

}  // namespace

// Stage a 128 x 64 tile of a K-major BF16 matrix (rows r0.., columns k0..) into the canonical
// layout at `dst`.  Rows >= rows_valid read zeros (cp.async with a 0-byte source).
__device__ __forceinline__ void load_tile(unsigned dst, const __nv_bfloat16 *src, int ld, int r0,
                                          int rows_valid, int k0, int tid) {
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int c = tid + q * 128;          // 1024 16-byte chunks: row = c / 8, chunk = c % 8
        const int r = c >> 3, kc = c & 7;
        const unsigned d = dst + (unsigned)((r >> 3) * 1024 + kc * 128 + (r & 7) * 16);
        const bool ok = r0 + r < rows_valid;
        const __nv_bfloat16 *s = src + (size_t)(ok ? r0 + r : 0) * ld + k0 + kc * 8;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(s), "r"(ok ? 16 : 0)
                     : "memory");
    }
}

__global__ void __launch_bounds__(128, 1)
tc_gemm_bf16_tn_kernel(int M, int N, int K, const __nv_bfloat16 *__restrict__ A, int lda,
                       const __nv_bfloat16 *__restrict__ B, int ldb, float *__restrict__ D, int ldd,
                       int k_per_slice, int mode, int *err) {
    extern __shared__ __align__(1024) unsigned char tsm[];
    __shared__ __align__(8) uint64_t bar[kStages];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    __shared__ int s_issued;   // stages whose MMAs were committed
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned base = (su32(tsm) + 1023u) & ~1023u;
    const int m0 = blockIdx.x * kTM, n0 = blockIdx.y * kTN;
    const int kb = blockIdx.z * k_per_slice;
    const int ke = min(K, kb + k_per_slice);
    const int nk = ke > kb ? (ke - kb) / kTK : 0;
    if (tid == 0) {
        s_fail = 0;
        s_issued = 0;
        for (int s = 0; s < kStages; s++) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&s_tmem)),
                     "r"(kTN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    // prologue: stages 0 .. kStages-2
#pragma unroll
    for (int s = 0; s < kStages - 1; s++) {
        if (s < nk) {
            const unsigned st = base + s * kStageBytes;
            load_tile(st, A, lda, m0, M, kb + s * kTK, tid);
            load_tile(st + kTileBytes, B, ldb, n0, N, kb + s * kTK, tid);
        }
        cpa_commit();
    }
    for (int kt = 0; kt < nk; kt++) {
        const int s = kt % kStages;
        cpa_wait<kStages - 2>();
        // make this thread's cp.async writes visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0 && !s_fail) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned st = base + s * kStageBytes;
#pragma unroll
            for (int kk = 0; kk < kTK / 16; kk++)
                umma(tmem, smem_desc(st + kk * 256), smem_desc(st + kTileBytes + kk * 256),
                     (kt > 0 || kk > 0) ? 1u : 0u);
            umma_commit(&bar[s]);
            s_issued = kt + 1;
        }
        // refill the stage consumed at kt - 1 once its MMAs are done
        const int nxt = kt + kStages - 1;
        if (nxt < nk) {
            const int sp = nxt % kStages;   // == (kt - 1) % kStages
            if (kt >= 1) {
                if (!mbar_wait(&bar[sp], (unsigned)(((kt - 1) / kStages) & 1))) {
                    if (lane == 0) s_fail = 1;
                }
            }
            __syncthreads();
            if (!s_fail) {
                const unsigned st = base + sp * kStageBytes;
                load_tile(st, A, lda, m0, M, kb + nxt * kTK, tid);
                load_tile(st + kTileBytes, B, ldb, n0, N, kb + nxt * kTK, tid);
            }
        }
        cpa_commit();
    }
    cpa_wait<0>();
    __syncthreads();
    // the last commit tracks every MMA this CTA issued
    const int issued = s_issued;
    bool ok = true;
    if (issued > 0) ok = mbar_wait(&bar[(issued - 1) % kStages], (unsigned)(((issued - 1) / kStages) & 1));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (!ok || s_fail) {
        if (tid == 0) atomicCAS(err, 0, 1);
    } else if (nk > 0) {
        // epilogue: warp w owns TMEM lanes (rows) 32w .. 32w+31
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < kTN; c0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
                "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                  "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                  "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
                  "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
                  "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
                float *drow = D + (size_t)row * ldd + n0 + c0;
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    if (n0 + c0 + j >= N) break;
                    const float x = __uint_as_float(v[j]);
                    if (mode == 0) drow[j] = x;
                    else atomicAdd(drow + j, x);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTN) : "memory");
}

bpf_status tc_gemm_bf16_tn(bpf_ctx *ctx, int M, int N, int K, const void *A, int lda, const void *B,
                           int ldb, float *D, int ldd, bool accumulate, int *err_dev, int splits) {
    if (M <= 0 || N <= 0 || K <= 0) return BPF_SUCCESS;
    if (K % kTK || lda % 8 || ldb % 8 || ((uintptr_t)A & 15) || ((uintptr_t)B & 15))
        return set_error(ctx, BPF_ERR_INVALID_VALUE,
                         "tensor-core GEMM: K (%d) must be a multiple of 64, leading dimensions of 8, "
                         "bases 16-byte aligned", K);
    const int mt = ceil_div(M, kTM), nt = ceil_div(N, kTN);
    if (splits <= 0) {   // enough K slices to fill the SMs (one CTA per SM), >= 4 tiles each
        const int want = std::max(1, (2 * ctx->num_sms) / std::max(1, mt * nt));
        splits = std::max(1, std::min(want, K / (4 * kTK)));
    }
    int kps = ceil_div(ceil_div(K, splits), kTK) * kTK;
    splits = ceil_div(K, kps);
    const int mode = (accumulate || splits > 1) ? 1 : 0;
    if (!accumulate && splits > 1)
        BPF_CUDA(ctx, cudaMemsetAsync(D, 0, sizeof(float) * (size_t)ldd * M, ctx->stream));
    BPF_CUDA(ctx, cudaFuncSetAttribute(tc_gemm_bf16_tn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmemBytes));
    KScope ks(ctx, BPF_KC_MLP, 2.0 * ((double)M * K + (double)N * K) + 4.0 * M * N,
              2.0 * (double)M * N * K);
    tc_gemm_bf16_tn_kernel<<<dim3(mt, nt, splits), 128, kSmemBytes, ctx->stream>>>(
        M, N, K, (const __nv_bfloat16 *)A, lda, (const __nv_bfloat16 *)B, ldb, D, ldd, kps, mode, err_dev);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

}  // namespace bpf

using namespace bpf;

extern "C" bpf_status bpf_tc_gemm_bf16(bpf_ctx *ctx, int M, int N, int K, const void *A, int lda,
                                      const void *B, int ldb, float *D, int ldd, int accumulate,
                                      int splits) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    if (M < 0 || N < 0 || K < 0 || (M > 0 && N > 0 && K > 0 && (!A || !B || !D)))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "tc_gemm_bf16: invalid argument");
    if (ldd < N || lda < K || ldb < K) return set_error(ctx, BPF_ERR_DIMENSION, "tc_gemm_bf16: leading dimension");
    bpf_status s;
    int *err = (int *)ws_get(ctx, WS_FLAGS, sizeof(int) * 4, &s);
    if (!err) return s;
    BPF_CUDA(ctx, cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    BPF_TRY(tc_gemm_bf16_tn(ctx, M, N, K, A, lda, B, ldb, D, ldd, accumulate != 0, err, splits));
    int h = 0;
    BPF_CUDA(ctx, cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h) return set_error(ctx, BPF_ERR_TIMEOUT, "tc_gemm_bf16: a tensor-core pipeline wait timed out");
    return BPF_SUCCESS;
}
