// CSR SpMM on row-major (RHS-interleaved) blocks, and the column-major <-> row-major
// conversions at the API boundary.
//
// Replaces mul!(W, A, P) (src/block_gmres.jl:299, :220,268; src/block_bicgstab.jl:135,145,
// 252,264), which CUDA.jl maps to cusparseSpMM on column-major blocks.  Here the block is
// stored row-major (the p values of one unknown are contiguous), so every nonzero a_ij
// gathers one contiguous p-vector of X: a group of G lanes per row reads it with coalesced
// loads while the row's (col, val) pairs are loaded once per group and broadcast by shuffles.
//
// Algorithmic bytes per launch: 12*nnz + 4*(n+1) + 8*n*p (X) + 8*n*p (Y written)
// [+ 8*n*p when beta != 0 or the residual form reads B].
#include <cstdint>
#include <type_traits>

#include "bpf_internal.cuh"

namespace bpf {

template <int G, int CPL, typename TX>
__global__ void __launch_bounds__(256)
spmm_rm_kernel(int n, const int *__restrict__ rp, const int *__restrict__ ci,
               const double *__restrict__ av, int base, int p, double alpha,
               const TX *__restrict__ X, double beta, double *__restrict__ Y,
               const double *__restrict__ Bres, const int *gate) {
    // one decision per CTA: the gate (st->active) may be cleared by the other stream mid-launch
    __shared__ int s_off;
    if (threadIdx.x == 0) s_off = (gate && *gate == 0) ? 1 : 0;
    __syncthreads();
    if (s_off) return;
    const int lane = threadIdx.x & 31;
    const int glane = lane % G;                    // lane within the row group
    const int groups_per_block = blockDim.x / G;
    const int grp = blockIdx.x * groups_per_block + threadIdx.x / G;
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane / G * G));
    for (int row = grp; row < n; row += gridDim.x * groups_per_block) {
        double acc[CPL];
#pragma unroll
        for (int j = 0; j < CPL; j++) acc[j] = 0.0;
        const int rs = __ldg(rp + row) - base, re = __ldg(rp + row + 1) - base;
        for (int kb = rs; kb < re; kb += G) {
            int k = kb + glane;
            int c = 0;
            double a = 0.0;
            if (k < re) {
                c = __ldg(ci + k) - base;
                a = __ldg(av + k);
            }
            const int cnt = min(G, re - kb);
            #pragma unroll 4   // several entries' loads in flight; same summation order
            for (int t = 0; t < cnt; t++) {
                const int ct = __shfl_sync(gmask, c, t, G);
                const double at = __shfl_sync(gmask, a, t, G);
                const TX *xr = X + (size_t)ct * p;
#pragma unroll
                for (int j = 0; j < CPL; j++) {
                    const int col = glane + j * G;
                    if (col < p) acc[j] += at * (double)__ldg(xr + col);
                }
            }
        }
        double *yr = Y + (size_t)row * p;
#pragma unroll
        for (int j = 0; j < CPL; j++) {
            const int col = glane + j * G;
            if (col < p) {
                double v;
                if (Bres) {
                    v = Bres[(size_t)row * p + col] - acc[j];
                } else {
                    v = alpha * acc[j];
                    if (beta != 0.0) v += beta * yr[col];
                }
                yr[col] = v;
            }
        }
    }
}

// Blocks of 64, 128, ... columns: a warp per row, lane l holding columns 2l, 2l + 1 (+ 64 j) as
// one 16-byte load per gathered row segment, half the load instructions of the 8-byte form and
// twice the bytes each one brings; eight entries' loads in flight.  Same products and summation
// order per output as spmm_rm_kernel.
template <int C2>
__global__ void __launch_bounds__(256)
spmm_rm2_kernel(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                const double *__restrict__ av, int base, int p, double alpha,
                const double *__restrict__ X, double beta, double *__restrict__ Y,
                const double *__restrict__ Bres, const int *gate) {
    __shared__ int s_off;
    if (threadIdx.x == 0) s_off = (gate && *gate == 0) ? 1 : 0;
    __syncthreads();
    if (s_off) return;
    const int lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < n; row += gridDim.x * warps) {
        double2 acc[C2];
#pragma unroll
        for (int j = 0; j < C2; j++) acc[j] = make_double2(0.0, 0.0);
        const int rs = __ldg(rp + row) - base, re = __ldg(rp + row + 1) - base;
        for (int kb = rs; kb < re; kb += 32) {
            const int k = kb + lane;
            int c = 0;
            double a = 0.0;
            if (k < re) {
                c = __ldg(ci + k) - base;
                a = __ldg(av + k);
            }
            const int cnt = min(32, re - kb);
#pragma unroll 8
            for (int t = 0; t < cnt; t++) {
                const int ct = __shfl_sync(0xffffffffu, c, t);
                const double at = __shfl_sync(0xffffffffu, a, t);
                const double2 *xr = reinterpret_cast<const double2 *>(X + (size_t)ct * p);
#pragma unroll
                for (int j = 0; j < C2; j++) {
                    const double2 v = __ldg(xr + lane + 32 * j);
                    acc[j].x += at * v.x;
                    acc[j].y += at * v.y;
                }
            }
        }
        double2 *yr = reinterpret_cast<double2 *>(Y + (size_t)row * p);
#pragma unroll
        for (int j = 0; j < C2; j++) {
            double2 v;
            if (Bres) {
                const double2 b = reinterpret_cast<const double2 *>(Bres + (size_t)row * p)[lane + 32 * j];
                v = make_double2(b.x - acc[j].x, b.y - acc[j].y);
            } else {
                v = make_double2(alpha * acc[j].x, alpha * acc[j].y);
                if (beta != 0.0) {
                    const double2 y0 = yr[lane + 32 * j];
                    v.x += beta * y0.x;
                    v.y += beta * y0.y;
                }
            }
            yr[lane + 32 * j] = v;
        }
    }
}

template <int C2>
static bpf_status launch_spmm2(bpf_ctx *ctx, int n, long long nnz, const int *rp, const int *ci,
                               const double *av, int base, int p, double alpha, const double *X,
                               double beta, double *Y, const double *B, const int *gate) {
    const int threads = 256, rows_per_block = threads / 32;
    int blocks = (int)std::min<long long>(ceil_div(n, rows_per_block), (long long)ctx->num_sms * 16);
    if (blocks < 1) blocks = 1;
    const double np = (double)n * p;
    const double bytes = 12.0 * nnz + 4.0 * (n + 1) + 8.0 * np + 8.0 * np + ((B || beta != 0.0) ? 8.0 * np : 0.0);
    KScope ks(ctx, BPF_KC_SPMM, bytes, 2.0 * nnz * p);
    spmm_rm2_kernel<C2><<<blocks, threads, 0, ctx->stream>>>(n, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

template <int G, int CPL, typename TX>
static bpf_status launch_spmm(bpf_ctx *ctx, int n, long long nnz, const int *rp, const int *ci,
                              const double *av, int base, int p, double alpha, const TX *X,
                              double beta, double *Y, const double *B, const int *gate) {
    const int threads = 256;
    const int groups = threads / G;
    long long blocks_needed = ceil_div(n, groups);
    int blocks = (int)std::min<long long>(blocks_needed, (long long)ctx->num_sms * 16);
    if (blocks < 1) blocks = 1;
    const double np = (double)n * p;
    const double bytes = 12.0 * nnz + 4.0 * (n + 1) + sizeof(TX) * np + 8.0 * np +
                         ((B || beta != 0.0) ? 8.0 * np : 0.0);
    KScope ks(ctx, BPF_KC_SPMM, bytes, 2.0 * nnz * p);
    spmm_rm_kernel<G, CPL, TX><<<blocks, threads, 0, ctx->stream>>>(n, rp, ci, av, base, p, alpha,
                                                                    X, beta, Y, B, gate);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

template <typename TX>
static bpf_status spmm_dispatch(bpf_ctx *ctx, int n, long long nnz, const int *rp, const int *ci,
                                const double *av, int base, int p, double alpha, const TX *X,
                                double beta, double *Y, const double *B, const int *gate) {
    if (n == 0 || p == 0) return BPF_SUCCESS;
    if constexpr (std::is_same<TX, double>::value) {
        // 16-byte rows: p a multiple of 64 and every block 16-byte aligned
        const bool aligned = ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y) |
                               reinterpret_cast<uintptr_t>(B)) & 15) == 0;
        if (aligned && p % 64 == 0 && p <= 256) {
            if (p == 64) return launch_spmm2<1>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
            if (p == 128) return launch_spmm2<2>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
            if (p == 192) return launch_spmm2<3>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
            return launch_spmm2<4>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
        }
    }
    if (p <= 4) return launch_spmm<4, 1>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
    if (p <= 8) return launch_spmm<8, 1>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
    if (p <= 16) return launch_spmm<16, 1>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
    if (p <= 32) return launch_spmm<32, 1>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
    if (p <= 64) return launch_spmm<32, 2>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
    if (p <= 128) return launch_spmm<32, 4>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
    if (p <= 256) return launch_spmm<32, 8>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
    return launch_spmm<32, 16>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
}

bpf_status spmm_rowmajor(bpf_ctx *ctx, int n, long long nnz, const int *rp, const int *ci,
                         const double *av, int base, int p, double alpha, const double *X,
                         double beta, double *Y, const double *B, const int *gate) {
    if (p > 512) {
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "spmm: p=%d > 512 right-hand sides", p);
    }
    return spmm_dispatch<double>(ctx, n, nnz, rp, ci, av, base, p, alpha, X, beta, Y, B, gate);
}

bpf_status spmm_rowmajor_f32x(bpf_ctx *ctx, int n, long long nnz, const int *rp, const int *ci,
                              const double *av, int base, int p, const float *X, double *Y,
                              const int *gate) {
    if (p > 512) {
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "spmm: p=%d > 512 right-hand sides", p);
    }
    return spmm_dispatch<float>(ctx, n, nnz, rp, ci, av, base, p, 1.0, X, 0.0, Y, nullptr, gate);
}

// ------------------------------------------------------------------------------------
// layout conversions (32x32 tiles through shared memory)
// ------------------------------------------------------------------------------------
__global__ void cm_to_rm_kernel(int n, int p, const double *__restrict__ src, int ld,
                                double *__restrict__ dst) {
    __shared__ double tile[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int c = c0 + j, r = r0 + threadIdx.x;
        if (r < n && c < p) tile[j][threadIdx.x] = src[(size_t)c * ld + r];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int r = r0 + j, c = c0 + threadIdx.x;
        if (r < n && c < p) dst[(size_t)r * p + c] = tile[threadIdx.x][j];
    }
}

__global__ void rm_to_cm_kernel(int n, int p, const double *__restrict__ src,
                                double *__restrict__ dst, int ld) {
    __shared__ double tile[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int r = r0 + j, c = c0 + threadIdx.x;
        if (r < n && c < p) tile[j][threadIdx.x] = src[(size_t)r * p + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int c = c0 + j, r = r0 + threadIdx.x;
        if (r < n && c < p) dst[(size_t)c * ld + r] = tile[threadIdx.x][j];
    }
}

bpf_status colmajor_to_rowmajor(bpf_ctx *ctx, int n, int p, const double *src, int ld,
                                double *dst) {
    if (n == 0 || p == 0) return BPF_SUCCESS;
    dim3 grid(ceil_div(n, 32), ceil_div(p, 32)), block(32, 8);
    cm_to_rm_kernel<<<grid, block, 0, ctx->stream>>>(n, p, src, ld, dst);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

bpf_status rowmajor_to_colmajor(bpf_ctx *ctx, int n, int p, const double *src, double *dst,
                                int ld) {
    if (n == 0 || p == 0) return BPF_SUCCESS;
    dim3 grid(ceil_div(n, 32), ceil_div(p, 32)), block(32, 8);
    rm_to_cm_kernel<<<grid, block, 0, ctx->stream>>>(n, p, src, dst, ld);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

}  // namespace bpf
