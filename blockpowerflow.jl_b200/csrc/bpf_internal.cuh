// Internal definitions shared by the libbpf translation units (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/bpf.h"

namespace bpf {

// ------------------------------------------------------------------------------------
// device-side error word (one per context)
// ------------------------------------------------------------------------------------
enum DevErr : int {
    DEV_OK = 0,
    DEV_ZERO_PIVOT = 1,      // factorization met a zero / non-positive pivot (row in aux)
    DEV_BARRIER_TIMEOUT = 2, // a bounded grid-barrier wait gave up
    DEV_NONFINITE = 3,       // NaN/Inf residual
    DEV_CHOL_FAIL = 4,       // Cholesky-QR Gram matrix not positive definite
};

struct DevStatus {
    int err;        // DevErr
    int aux;        // row / column index for diagnostics
    unsigned bar_count;  // grid barrier arrival counter
    unsigned bar_gen;    // grid barrier generation
    long long wait_limit;  // polls before a grid barrier gives up (<= 0: kSpinLimit); kept by resets
    int pad[2];
};

// Workspace slots held by a context (grow-only, reused across calls).
enum Slot : int {
    WS_PARTIAL = 0,   // split-K partial sums of Gram products
    WS_SMALL,         // p x p scratch matrices
    WS_A,
    WS_B,
    WS_C,
    WS_D,
    WS_E,
    WS_F,
    WS_G,
    WS_H,
    WS_V,             // Krylov basis
    WS_HESS,          // packed R blocks of the block Hessenberg QR
    WS_STATE,         // solver state struct
    WS_HIST,          // residual history
    WS_I32,
    WS_NORM,          // reduction partials
    WS_Z,             // least-squares right-hand side blocks
    WS_HY,            // Householder reflectors (2p x p) and T factors per block column
    WS_HSCR,          // scratch of the one-CTA small-matrix kernels
    WS_VEC,           // n x p working blocks of a solve
    WS_Y,             // block back-substitution result Y
    WS_ZB,            // flexible GMRES: preconditioned basis blocks
    WS_FLAGS,         // small device status words (tensor-core GEMM errors)
    WS_DEFL,          // deflated block-GMRES: Q_C, Z R^{-1}, E_j blocks
    WS_COUNT
};

}  // namespace bpf

struct bpf_ctx {
    cudaStream_t stream = nullptr;
    int device = 0;
    int num_sms = 148;
    int max_smem_optin = 0;
    std::string last_error;
    long long launches = 0;
    // FP64 block products on the tensor pipe (DMMA) instead of FMA; BPF_FP64_MMA=0 turns it
    // off (used to compare the two paths).
    bool fp64_mma = true;
    // Second (high-priority) stream on which block-GMRES runs the Hessenberg QR update of
    // iteration k while the main stream runs the Arnoldi step of iteration k+1; events hand
    // the C blocks over (ev_a) and back (ev_b), double buffered by iteration parity.
    // BPF_OVERLAP=0 keeps everything on the main stream.
    bool overlap = true;
    cudaStream_t hstream = nullptr;
    cudaEvent_t ev_a[2] = {nullptr, nullptr};
    cudaEvent_t ev_b[2] = {nullptr, nullptr};
    // per-kernel-class event timing (bpf_ctx_set_timing)
    bool timing = false;
    std::vector<cudaEvent_t> event_pool;
    size_t event_next = 0;
    struct TimedLaunch { int kc; cudaEvent_t a, b; double bytes, flops; };
    std::vector<TimedLaunch> timed;
    bpf::DevStatus *dstat = nullptr;   // device
    bpf::DevStatus *hstat = nullptr;   // pinned host mirror
    void *ws[bpf::WS_COUNT] = {};
    size_t ws_bytes[bpf::WS_COUNT] = {};
};

namespace bpf {

// ------------------------------------------------------------------------------------
// host-side error helpers
// ------------------------------------------------------------------------------------
bpf_status set_error(bpf_ctx *ctx, bpf_status st, const char *fmt, ...);
// A library context was created on `dev`: bpf_prec_apply_noalloc looks its static scratch's
// address up again on its next call there (noalloc.cu).
void noalloc_forget_device(int dev);
bpf_status cuda_error(bpf_ctx *ctx, cudaError_t e, const char *what, const char *file, int line);
void *ws_get(bpf_ctx *ctx, int slot, size_t bytes, bpf_status *st);
bpf_status check_dev_status(bpf_ctx *ctx, const char *where);
bpf_status reset_dev_status(bpf_ctx *ctx);

#define BPF_CUDA(ctx, call)                                                          \
    do {                                                                             \
        cudaError_t _e = (call);                                                     \
        if (_e != cudaSuccess) return ::bpf::cuda_error(ctx, _e, #call, __FILE__, __LINE__); \
    } while (0)

#define BPF_LAUNCHED(ctx)                                                            \
    do {                                                                             \
        (ctx)->launches++;                                                           \
        cudaError_t _e = cudaGetLastError();                                         \
        if (_e != cudaSuccess) return ::bpf::cuda_error(ctx, _e, "kernel launch", __FILE__, __LINE__); \
    } while (0)

#define BPF_TRY(expr)                                                                \
    do {                                                                             \
        bpf_status _s = (expr);                                                      \
        if (_s != BPF_SUCCESS) return _s;                                            \
    } while (0)

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Records a CUDA event pair around one launch when the context's timing is on.  A launch
// gated on a device flag (it returns at once unless a rare condition was raised) is not
// recorded (gated = true): its algorithmic bytes and flops would count work it skips, so the
// class totals cover the launches that always do their work.
cudaEvent_t timing_event(bpf_ctx *ctx);
struct KScope {
    bpf_ctx *ctx;
    int kc;
    double bytes, flops;
    cudaEvent_t a = nullptr;
    KScope(bpf_ctx *c, int k, double algo_bytes = 0.0, double algo_flops = 0.0, bool gated = false)
        : ctx(c), kc(k), bytes(algo_bytes), flops(algo_flops) {
        if (ctx->timing && !gated) {
            a = timing_event(ctx);
            if (a) cudaEventRecord(a, ctx->stream);
        }
    }
    ~KScope() {
        if (a) {
            cudaEvent_t b = timing_event(ctx);
            if (b) {
                cudaEventRecord(b, ctx->stream);
                ctx->timed.push_back({kc, a, b, bytes, flops});
            }
        }
    }
};

// Launches made while it lives go to stream `s` (restored on scope exit, error paths included).
struct StreamSwap {
    bpf_ctx *ctx;
    cudaStream_t saved;
    StreamSwap(bpf_ctx *c, cudaStream_t s) : ctx(c), saved(c->stream) { ctx->stream = s; }
    ~StreamSwap() { ctx->stream = saved; }
};

// ------------------------------------------------------------------------------------
// device helpers
// ------------------------------------------------------------------------------------
#ifdef __CUDACC__
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_i32(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Spin limit of every cross-CTA wait: ~2^21 polls with a short sleep each (about a second),
// after which the wait records DEV_BARRIER_TIMEOUT and returns.
constexpr long long kSpinLimit = 1LL << 21;

// Grid-wide barrier for a cooperative (co-resident) launch.  `gen` is the generation the
// calling block last saw (read once at kernel start by thread 0 of each block).  Returns
// false (in every thread of the block) if the barrier timed out or an error is pending, in
// which case the caller must return without further global writes.  A waiting block gives up
// after the context's wait limit (ds->wait_limit polls, kSpinLimit when not set).
__device__ __forceinline__ bool grid_barrier(DevStatus *ds, unsigned &gen) {
    __shared__ int s_ok;
    __syncthreads();
    if (gridDim.x == 1) {
        return true;
    }
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned g = gen;
        __threadfence();
        unsigned prev = atomicAdd(&ds->bar_count, 1u);
        if (prev == gridDim.x - 1) {
            atomicExch(&ds->bar_count, 0u);
            __threadfence();
            st_release_u32(&ds->bar_gen, g + 1);
        } else {
            long long it = 0;
            const long long lim = ds->wait_limit > 0 ? ds->wait_limit : kSpinLimit;
            while (ld_acquire_u32(&ds->bar_gen) == g) {
                if (++it > lim || ld_relaxed_i32(&ds->err) != 0) {
                    ok = 0;
                    atomicCAS(&ds->err, 0, (int)DEV_BARRIER_TIMEOUT);
                    break;
                }
                __nanosleep(64);
            }
        }
        gen = g + 1;
        if (ld_relaxed_i32(&ds->err) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ unsigned barrier_gen_start(DevStatus *ds) {
    return ld_acquire_u32(&ds->bar_gen);
}
#endif

// ------------------------------------------------------------------------------------
// launchers implemented in the .cu files
// ------------------------------------------------------------------------------------
// Column-major (ld) <-> row-major (n x p, ld = p) block conversions.
bpf_status colmajor_to_rowmajor(bpf_ctx *ctx, int n, int p, const double *src, int ld,
                                double *dst);
bpf_status rowmajor_to_colmajor(bpf_ctx *ctx, int n, int p, const double *src, double *dst,
                                int ld);

// CSR SpMM on row-major blocks: Y = alpha*A*X + beta*Y, or (residual) Y = B - A*X when
// B != nullptr.  base = index base of the CSR arrays.
bpf_status spmm_rowmajor(bpf_ctx *ctx, int n, long long nnz, const int *rp, const int *ci,
                         const double *av, int base, int p, double alpha, const double *X,
                         double beta, double *Y, const double *B, const int *gate = nullptr);
// Same with an FP32 input block (mixed-precision path): Y = A*X.
bpf_status spmm_rowmajor_f32x(bpf_ctx *ctx, int n, long long nnz, const int *rp, const int *ci,
                              const double *av, int base, int p, const float *X, double *Y,
                              const int *gate = nullptr);

}  // namespace bpf
