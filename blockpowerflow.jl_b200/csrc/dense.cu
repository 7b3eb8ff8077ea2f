// Dense block kernels: Gram products, tall x small products, Cholesky-QR, reductions.
//
// They replace the cuBLAS gemm / nrm2 / dot and cuSOLVER geqrf / orgqr calls the reference
// makes on n x p blocks (src/block_gmres.jl:301-316, src/block_utils.jl:46-53,
// src/block_bicgstab.jl:136-153).  FP64 throughout (B200 runs FP64 FMA and FP64 MMA at the
// same rate, so the FMA path with shared-memory tiles is used).
//
//  gram : Out_j = A_j^T B, split over rows into chunks (grid.x), one p x p tile per CTA,
//         partial sums reduced by a second deterministic kernel.
//         Algorithmic bytes: 8*n*p*(nb + 1); flops 2*n*p*p*nb.
//  tsmm : Out = beta*C + alpha*sum_j A_j S_j, one 64-row x 64-column tile per CTA.
//         Algorithmic bytes: 8*n*p*(nb + 1 [+1 for C]); flops 2*n*p*p*nb.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "bpf_internal.cuh"
#include "dense.cuh"
#include "small.cuh"

namespace bpf {

constexpr int kGramRows = 32;   // rows per shared-memory stage of gram
constexpr int kTsmmRows = 64;   // rows per CTA of tsmm
constexpr int kTsmmK = 16;      // inner-dimension stage of tsmm

__device__ __forceinline__ bool gate_off(const SolveState *st, const int *gate,
                                         const int *gate2 = nullptr) {
    if (st && !st->active) return true;
    if (gate && *gate == 0) return true;
    if (gate2 && *gate2 == 0) return true;
    return false;
}

// The gate decided once per CTA (thread 0 reads it): st->active is cleared by the Hessenberg
// update on the other stream, possibly between the reads of two warps, and warps that disagreed
// would leave some of the CTA past a barrier the others never reach.
__device__ __forceinline__ bool cta_gate_off(const SolveState *st, const int *gate, const int *gate2 = nullptr) {
    __shared__ int s_off;
    if (threadIdx.x == 0) s_off = gate_off(st, gate, gate2) ? 1 : 0;
    __syncthreads();
    return s_off != 0;
}


// ---------------------------------------------------------------------------------------
// gram
// ---------------------------------------------------------------------------------------
template <int GT>
__global__ void __launch_bounds__(256)
gram_partial_kernel(int n, int p, int nb, const double *__restrict__ A, size_t strideA,
                    const double *__restrict__ B, double *__restrict__ partial,
                    int rows_per_chunk, const SolveState *st, const int *gate,
                    const int *gate2) {
    if (cta_gate_off(st, gate, gate2)) return;
    constexpr int TPD = GT / 16;   // outputs per thread per dimension
    __shared__ double As[kGramRows][GT];
    __shared__ double Bs[kGramRows][GT];
    const int chunk = blockIdx.x, j = blockIdx.y;
    const int ntile = (p + GT - 1) / GT;
    const int a0 = (blockIdx.z / ntile) * GT, b0 = (blockIdx.z % ntile) * GT;
    const int r_begin = chunk * rows_per_chunk;
    const int r_end = min(n, r_begin + rows_per_chunk);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const double *Aj = A + (size_t)j * strideA;
    double acc[TPD][TPD];
#pragma unroll
    for (int i = 0; i < TPD; i++)
#pragma unroll
        for (int k = 0; k < TPD; k++) acc[i][k] = 0.0;
    for (int r0 = r_begin; r0 < r_end; r0 += kGramRows) {
        for (int e = threadIdx.x; e < kGramRows * GT; e += 256) {
            const int rr = e / GT, cc = e % GT, r = r0 + rr;
            const bool rok = r < r_end;
            As[rr][cc] = (rok && a0 + cc < p) ? __ldg(Aj + (size_t)r * p + a0 + cc) : 0.0;
            Bs[rr][cc] = (rok && b0 + cc < p) ? __ldg(B + (size_t)r * p + b0 + cc) : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < kGramRows; rr++) {
            double a[TPD], b[TPD];
#pragma unroll
            for (int i = 0; i < TPD; i++) a[i] = As[rr][ty + 16 * i];
#pragma unroll
            for (int k = 0; k < TPD; k++) b[k] = Bs[rr][tx + 16 * k];
#pragma unroll
            for (int i = 0; i < TPD; i++)
#pragma unroll
                for (int k = 0; k < TPD; k++) acc[i][k] = fma(a[i], b[k], acc[i][k]);
        }
        __syncthreads();
    }
    double *out = partial + ((size_t)chunk * nb + j) * p * p;
#pragma unroll
    for (int i = 0; i < TPD; i++) {
        const int a = a0 + ty + 16 * i;
        if (a >= p) continue;
#pragma unroll
        for (int k = 0; k < TPD; k++) {
            const int b = b0 + tx + 16 * k;
            if (b < p) out[(size_t)a * p + b] = acc[i][k];
        }
    }
}

__global__ void gram_reduce_kernel(int total, int nchunks, const double *__restrict__ partial,
                                   double *__restrict__ out, double alpha, int accumulate,
                                   double *__restrict__ out2, const SolveState *st,
                                   const int *gate, const int *gate2) {
    if (cta_gate_off(st, gate, gate2)) return;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < nchunks; c++) s += partial[(size_t)c * total + e];
        s *= alpha;
        if (out2) out2[e] = s;
        if (accumulate) s += out[e];
        out[e] = s;
    }
}

template <int GT>
__global__ void gram_dmma_cl_kernel(int n, int p, int nb, const double *__restrict__ A,
                                    size_t strideA, const double *__restrict__ B,
                                    double *__restrict__ partial, int rows_per_chunk,
                                    const SolveState *st, const int *gate, const int *gate2);
// Epilogue of gram_pipe_kernel when the row chunks of a block form a single cluster: the
// cluster's sum is the result (Out = alpha * sum [+ Out], Out2 = alpha * sum).
struct GramEpilogue {
    int direct;
    int accumulate;
    double alpha;
    double *out;
    double *out2;
};
__global__ void
gram_pipe_kernel(int n, int p, int nb, const double *__restrict__ A, size_t strideA,
                 const double *__restrict__ B, double *__restrict__ partial, int rows_per_chunk,
                 const SolveState *st, const int *gate, const int *gate2, GramEpilogue ep);
static bool pipe_ok(int p, const void *A, size_t strideA, const void *B, size_t strideB);
extern const size_t kGramPipeSmemBytes;

bpf_status gram(bpf_ctx *ctx, int n, int p, int nb, const double *A, size_t strideA,
                const double *B, double *Out, double alpha, bool accumulate,
                const SolveState *st, const int *qr_gate, double *Out2, const int *gate2) {
    if (nb <= 0 || p <= 0) return BPF_SUCCESS;
    const int GT = p <= 16 ? 16 : (p <= 32 ? 32 : 64);
    const int ntile = ceil_div(p, GT);
    const int tiles = ntile * ntile;
    bpf_status s;
    if (ctx->fp64_mma && GT == 64 && pipe_ok(p, A, strideA, B, 0)) {
        // One wave of resident CTAs (two per SM): the cluster size cs and the number of
        // clusters per block are picked so that cs * ncl * nb * tiles fits it, with at least
        // 128 rows per CTA; a block covered by one cluster skips the partial-sum pass.
        const int slots = 2 * ctx->num_sms;
        const int units = nb * tiles;
        int cs = 8;
        while (cs > 1 && cs * units > slots) cs >>= 1;
        int ncl = std::max(1, slots / (cs * units));
        ncl = std::max(1, std::min(ncl, n / (cs * 128)));
        const int pchunks = cs * ncl;
        int rpc = ceil_div(std::max(n, 1), pchunks);
        rpc = ceil_div(rpc, 32) * 32;
        const bool direct = ncl == 1;
        double *part2 = nullptr;
        if (!direct) {
            part2 = (double *)ws_get(ctx, WS_PARTIAL, sizeof(double) * (size_t)ncl * nb * p * p, &s);
            if (!part2) return s;
        }
        KScope ks(ctx, BPF_KC_GRAM, 8.0 * n * p * (nb + (A == B ? 0 : 1)), 2.0 * n * p * (double)p * nb,
                  qr_gate != nullptr || gate2 != nullptr);
        BPF_CUDA(ctx, cudaFuncSetAttribute(gram_pipe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kGramPipeSmemBytes));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(pchunks, nb, tiles);
        cfg.blockDim = dim3(256, 1, 1);
        cfg.dynamicSmemBytes = kGramPipeSmemBytes;
        cfg.stream = ctx->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cs;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        GramEpilogue ep{direct ? 1 : 0, accumulate ? 1 : 0, alpha, Out, Out2};
        BPF_CUDA(ctx, cudaLaunchKernelEx(&cfg, gram_pipe_kernel, n, p, nb, A, strideA, B, part2, rpc,
                                         st, qr_gate, gate2, ep));
        BPF_LAUNCHED(ctx);
        if (!direct) {
            const int total = nb * p * p;
            const int blocks = std::min(ceil_div(total, 256), ctx->num_sms * 4);
            gram_reduce_kernel<<<blocks, 256, 0, ctx->stream>>>(total, ncl, part2, Out, alpha,
                                                                 accumulate ? 1 : 0, Out2, st, qr_gate, gate2);
            BPF_LAUNCHED(ctx);
        }
        return BPF_SUCCESS;
    }
    const int target = ctx->num_sms * 4;
    int nchunks = std::max(1, std::min(ceil_div(n, kGramRows), target / std::max(1, nb * tiles)));
    int rows_per_chunk = ceil_div(std::max(n, 1), nchunks);
    rows_per_chunk = ceil_div(rows_per_chunk, kGramRows) * kGramRows;
    nchunks = std::max(1, ceil_div(std::max(n, 1), rows_per_chunk));
    // DMMA path: chunks in clusters of 8 (trailing chunks of the last cluster may be empty),
    // one partial per cluster
    const bool cl = ctx->fp64_mma;
    const int nclusters = ceil_div(nchunks, 8);
    const int grid_x = cl ? 8 * nclusters : nchunks;
    const int nparts = cl ? nclusters : nchunks;
    double *partial = (double *)ws_get(ctx, WS_PARTIAL, sizeof(double) * (size_t)nparts * nb * p * p, &s);
    if (!partial) return s;
    dim3 grid(grid_x, nb, tiles);
    KScope ks(ctx, BPF_KC_GRAM, 8.0 * n * p * (nb + (A == B ? 0 : 1)), 2.0 * n * p * (double)p * nb,
              qr_gate != nullptr || gate2 != nullptr);
    if (cl) {
        if (GT == 16)
            gram_dmma_cl_kernel<16><<<grid, 128, 0, ctx->stream>>>(n, p, nb, A, strideA, B, partial,
                                                                    rows_per_chunk, st, qr_gate, gate2);
        else if (GT == 32)
            gram_dmma_cl_kernel<32><<<grid, 128, 0, ctx->stream>>>(n, p, nb, A, strideA, B, partial,
                                                                    rows_per_chunk, st, qr_gate, gate2);
        else
            gram_dmma_cl_kernel<64><<<grid, 128, 0, ctx->stream>>>(n, p, nb, A, strideA, B, partial,
                                                                    rows_per_chunk, st, qr_gate, gate2);
    } else if (GT == 16)
        gram_partial_kernel<16><<<grid, 256, 0, ctx->stream>>>(n, p, nb, A, strideA, B, partial,
                                                                rows_per_chunk, st, qr_gate, gate2);
    else if (GT == 32)
        gram_partial_kernel<32><<<grid, 256, 0, ctx->stream>>>(n, p, nb, A, strideA, B, partial,
                                                                rows_per_chunk, st, qr_gate, gate2);
    else
        gram_partial_kernel<64><<<grid, 256, 0, ctx->stream>>>(n, p, nb, A, strideA, B, partial,
                                                                rows_per_chunk, st, qr_gate, gate2);
    BPF_LAUNCHED(ctx);
    int total = nb * p * p;
    int blocks = std::min(ceil_div(total, 256), ctx->num_sms * 4);
    gram_reduce_kernel<<<blocks, 256, 0, ctx->stream>>>(total, nparts, partial, Out, alpha,
                                                         accumulate ? 1 : 0, Out2, st, qr_gate, gate2);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// ---------------------------------------------------------------------------------------
// FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) versions of gram and tsmm.
// Fragment layout of mma.sync.aligned.m8n8k4.row.col.f64: lane = 4 g + t, A[g][t],
// B[t][g], C[g][2t], C[g][2t+1].  Shared-memory rows are padded to a stride = 4 (mod 16)
// doubles so both half-warps read 16 distinct 8-byte banks.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Out tile GT x GT of A_j^T B over a chunk of rows; 4 warps in a 2 x 2 layout.
template <int GT>
__global__ void __launch_bounds__(128)
gram_dmma_kernel(int n, int p, int nb, const double *__restrict__ A, size_t strideA,
                 const double *__restrict__ B, double *__restrict__ partial, int rows_per_chunk,
                 const SolveState *st, const int *gate, const int *gate2) {
    if (cta_gate_off(st, gate, gate2)) return;
    constexpr int RS = 32, S = GT + 4, WT = GT / 2, MT = WT / 8;
    __shared__ double As[RS * S];
    __shared__ double Bs[RS * S];
    const int chunk = blockIdx.x, j = blockIdx.y;
    const int ntile = (p + GT - 1) / GT;
    const int a0 = (blockIdx.z / ntile) * GT, b0 = (blockIdx.z % ntile) * GT;
    const int r_begin = chunk * rows_per_chunk;
    const int r_end = min(n, r_begin + rows_per_chunk);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t4 = lane & 3;
    const double *Aj = A + (size_t)j * strideA;
    double acc[MT][MT][2];
#pragma unroll
    for (int mi = 0; mi < MT; mi++)
#pragma unroll
        for (int ni = 0; ni < MT; ni++) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
    for (int r0 = r_begin; r0 < r_end; r0 += RS) {
        for (int e = tid; e < RS * GT; e += 128) {
            const int rr = e / GT, cc = e % GT, r = r0 + rr;
            const bool rok = r < r_end;
            As[rr * S + cc] = (rok && a0 + cc < p) ? __ldg(Aj + (size_t)r * p + a0 + cc) : 0.0;
            Bs[rr * S + cc] = (rok && b0 + cc < p) ? __ldg(B + (size_t)r * p + b0 + cc) : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < RS / 4; ks++) {
            const int k = ks * 4 + t4;
            double a[MT], b[MT];
#pragma unroll
            for (int mi = 0; mi < MT; mi++) a[mi] = As[k * S + wm * WT + mi * 8 + g];
#pragma unroll
            for (int ni = 0; ni < MT; ni++) b[ni] = Bs[k * S + wn * WT + ni * 8 + g];
#pragma unroll
            for (int mi = 0; mi < MT; mi++)
#pragma unroll
                for (int ni = 0; ni < MT; ni++) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
        }
        __syncthreads();
    }
    double *out = partial + ((size_t)chunk * nb + j) * p * p;
#pragma unroll
    for (int mi = 0; mi < MT; mi++) {
        const int row = a0 + wm * WT + mi * 8 + g;
        if (row >= p) continue;
#pragma unroll
        for (int ni = 0; ni < MT; ni++) {
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int col = b0 + wn * WT + ni * 8 + 2 * t4 + i;
                if (col < p) out[(size_t)row * p + col] = acc[mi][ni][i];
            }
        }
    }
}

// Same product with the row chunks grouped in clusters of 8 CTAs: the 8 partial tiles are
// summed through distributed shared memory (each CTA of the cluster sums 1/8 of the tile's
// rows over the 8 CTAs) and one partial per cluster goes to global memory, an 8x cut of the
// partial-sum traffic.  A gated-off CTA does not return early: its peers read its shared memory
// in the cluster sum, and the gate (st->active, cleared by the Hessenberg update on the other
// stream) may read differently in two CTAs of one cluster; it runs no row stages and stores
// nothing (such a launch belongs to an iteration past the stopping point, whose results are
// discarded).
template <int GT>
__global__ void __cluster_dims__(8, 1, 1) __launch_bounds__(128)
gram_dmma_cl_kernel(int n, int p, int nb, const double *__restrict__ A, size_t strideA,
                    const double *__restrict__ B, double *__restrict__ partial,
                    int rows_per_chunk, const SolveState *st, const int *gate,
                    const int *gate2) {
    const bool off = cta_gate_off(st, gate, gate2);
    namespace cg = cooperative_groups;
    constexpr int RS = 32, S = GT + 4, WT = GT / 2, MT = WT / 8;
    __shared__ double sbuf[2 * RS * S];
    double *As = sbuf, *Bs = sbuf + RS * S;
    const int chunk = blockIdx.x, j = blockIdx.y;
    const int ntile = (p + GT - 1) / GT;
    const int a0 = (blockIdx.z / ntile) * GT, b0 = (blockIdx.z % ntile) * GT;
    const int r_begin = chunk * rows_per_chunk;
    const int r_end = off ? r_begin : min(n, r_begin + rows_per_chunk);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t4 = lane & 3;
    const double *Aj = A + (size_t)j * strideA;
    double acc[MT][MT][2];
#pragma unroll
    for (int mi = 0; mi < MT; mi++)
#pragma unroll
        for (int ni = 0; ni < MT; ni++) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
    for (int r0 = r_begin; r0 < r_end; r0 += RS) {
        for (int e = tid; e < RS * GT; e += 128) {
            const int rr = e / GT, cc = e % GT, r = r0 + rr;
            const bool rok = r < r_end;
            As[rr * S + cc] = (rok && a0 + cc < p) ? __ldg(Aj + (size_t)r * p + a0 + cc) : 0.0;
            Bs[rr * S + cc] = (rok && b0 + cc < p) ? __ldg(B + (size_t)r * p + b0 + cc) : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < RS / 4; ks++) {
            const int k = ks * 4 + t4;
            double a[MT], b[MT];
#pragma unroll
            for (int mi = 0; mi < MT; mi++) a[mi] = As[k * S + wm * WT + mi * 8 + g];
#pragma unroll
            for (int ni = 0; ni < MT; ni++) b[ni] = Bs[k * S + wn * WT + ni * 8 + g];
#pragma unroll
            for (int mi = 0; mi < MT; mi++)
#pragma unroll
                for (int ni = 0; ni < MT; ni++) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
        }
        __syncthreads();
    }
    // this CTA's tile into its shared memory (GT x GT, row-major)
#pragma unroll
    for (int mi = 0; mi < MT; mi++)
#pragma unroll
        for (int ni = 0; ni < MT; ni++)
#pragma unroll
            for (int i = 0; i < 2; i++)
                sbuf[(wm * WT + mi * 8 + g) * GT + wn * WT + ni * 8 + 2 * t4 + i] = acc[mi][ni][i];
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    const int rank = (int)cluster.block_rank();
    constexpr int RPR = GT / 8;   // tile rows summed by each CTA of the cluster
    double *out = partial + ((size_t)(chunk / 8) * nb + j) * p * p;
    for (int e = tid; e < RPR * GT; e += 128) {
        const int a = rank * RPR + e / GT, b = e % GT;
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 8; q++) s += cluster.map_shared_rank(sbuf, q)[a * GT + b];
        if (!off && a0 + a < p && b0 + b < p) out[(size_t)(a0 + a) * p + b0 + b] = s;
    }
    cluster.sync();
}

// Out rows r0..r0+63, columns b0..b0+GT-1 of beta*C + alpha*sum_j A_j S_j; 4 warps 2 x 2.
template <int GT>
__global__ void __launch_bounds__(128)
tsmm_dmma_kernel(int n, int p, int nb, const double *__restrict__ A, size_t strideA,
                 const double *__restrict__ S, size_t strideS, double alpha, const double *Cin,
                 double beta, double *Out, const SolveState *st, const int *nb_dev,
                 const int *gate, const int *gate2) {
    if (cta_gate_off(st, gate, gate2)) return;
    constexpr int KC = 32, SA = KC + 4, SB = GT + 4, WN = GT / 2, MTN = WN / 8;
    __shared__ double As[64 * SA];
    __shared__ double Bs[KC * SB];
    const int r0 = blockIdx.x * 64;
    const int b0 = blockIdx.y * GT;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t4 = lane & 3;
    int nbl = nb;
    if (nb_dev) nbl = min(nb, *nb_dev);
    double acc[4][MTN][2];
#pragma unroll
    for (int mi = 0; mi < 4; mi++)
#pragma unroll
        for (int ni = 0; ni < MTN; ni++) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
    for (int j = 0; j < nbl; j++) {
        const double *Aj = A + (size_t)j * strideA;
        const double *Sj = S + (size_t)j * strideS;
        for (int k0 = 0; k0 < p; k0 += KC) {
            for (int e = tid; e < 64 * KC; e += 128) {
                const int rr = e / KC, kk = e % KC;
                const int r = r0 + rr, c = k0 + kk;
                As[rr * SA + kk] = (r < n && c < p) ? __ldg(Aj + (size_t)r * p + c) : 0.0;
            }
            for (int e = tid; e < KC * GT; e += 128) {
                const int kk = e / GT, cc = e % GT;
                const int a = k0 + kk, b = b0 + cc;
                Bs[kk * SB + cc] = (a < p && b < p) ? __ldg(Sj + (size_t)a * p + b) : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int ks = 0; ks < KC / 4; ks++) {
                const int k = ks * 4 + t4;
                double a[4], b[MTN];
#pragma unroll
                for (int mi = 0; mi < 4; mi++) a[mi] = As[(wm * 32 + mi * 8 + g) * SA + k];
#pragma unroll
                for (int ni = 0; ni < MTN; ni++) b[ni] = Bs[k * SB + wn * WN + ni * 8 + g];
#pragma unroll
                for (int mi = 0; mi < 4; mi++)
#pragma unroll
                    for (int ni = 0; ni < MTN; ni++) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int mi = 0; mi < 4; mi++) {
        const int r = r0 + wm * 32 + mi * 8 + g;
        if (r >= n) continue;
#pragma unroll
        for (int ni = 0; ni < MTN; ni++) {
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int b = b0 + wn * WN + ni * 8 + 2 * t4 + i;
                if (b >= p) continue;
                double v = alpha * acc[mi][ni][i];
                if (Cin && beta != 0.0) v += beta * Cin[(size_t)r * p + b];
                Out[(size_t)r * p + b] = v;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Pipelined FP64 tensor-core products (p even, 32 < p, 64-wide output tiles): 8 warps in a
// 4 x 2 layout (16 x 32 outputs each), operands staged by 16-byte cp.async in a 3-stage ring
// so the loads of chunk c+2 are in flight while chunk c computes; padded row strides (36 and
// 68 doubles) keep the m8n8k4 fragment loads free of bank conflicts.  ~105 KB of shared
// memory per CTA, two CTAs per SM.
// ---------------------------------------------------------------------------------------
constexpr int kPipeStages = 3;

__device__ __forceinline__ void cp_async16_zfill(void *smem, const void *gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Out (rows r0..r0+63, columns b0..b0+63) = beta*Cin + alpha*sum_j A_j S_j.
__global__ void __launch_bounds__(256, 2)
tsmm_pipe_kernel(int n, int p, int nb, const double *__restrict__ A, size_t strideA,
                 const double *__restrict__ S, size_t strideS, double alpha, const double *Cin,
                 double beta, double *Out, const SolveState *st, const int *gate, const int *gate2) {
    if (cta_gate_off(st, gate, gate2)) return;
    constexpr int BM = 64, GT = 64, KC = 32, SA = KC + 4, SB = GT + 4, ST = kPipeStages;
    extern __shared__ __align__(16) double psm[];
    double *As = psm;                          // ST x BM x SA
    double *Bs = psm + ST * BM * SA;           // ST x KC x SB
    const int r0 = blockIdx.x * BM, b0 = blockIdx.y * GT;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t4 = lane & 3;
    const int kpb = (p + KC - 1) / KC;
    const int nchunks = nb * kpb;
    auto load = [&](int ch, int stage) {
        const int j = ch / kpb, k0 = (ch - j * kpb) * KC;
        const double *Aj = A + (size_t)j * strideA;
        const double *Sj = S + (size_t)j * strideS;
        double *as = As + stage * BM * SA;
        double *bs = Bs + stage * KC * SB;
#pragma unroll
        for (int q = 0; q < BM * KC / 2 / 256; q++) {
            const int e = tid + q * 256;
            const int rr = e / (KC / 2), cc = (e % (KC / 2)) * 2;
            const int r = r0 + rr, c = k0 + cc;
            const bool ok = r < n && c < p;
            cp_async16_zfill(as + rr * SA + cc, ok ? Aj + (size_t)r * p + c : Aj, ok ? 16 : 0);
        }
#pragma unroll
        for (int q = 0; q < KC * GT / 2 / 256; q++) {
            const int e = tid + q * 256;
            const int kk = e / (GT / 2), cc = (e % (GT / 2)) * 2;
            const int a = k0 + kk, b = b0 + cc;
            const bool ok = a < p && b < p;
            cp_async16_zfill(bs + kk * SB + cc, ok ? Sj + (size_t)a * p + b : Sj, ok ? 16 : 0);
        }
    };
    double acc[2][4][2];
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
#pragma unroll
    for (int s0 = 0; s0 < ST - 1; s0++) {
        if (s0 < nchunks) load(s0, s0);
        cp_async_commit_group();
    }
    for (int ch = 0; ch < nchunks; ch++) {
        cp_async_wait_group<ST - 2>();
        __syncthreads();
        const int nxt = ch + ST - 1;   // its stage was consumed at iteration ch - 1
        if (nxt < nchunks) load(nxt, nxt % ST);
        cp_async_commit_group();
        const double *as = As + (ch % ST) * BM * SA;
        const double *bs = Bs + (ch % ST) * KC * SB;
#pragma unroll
        for (int ks = 0; ks < KC / 4; ks++) {
            const int k = ks * 4 + t4;
            double a[2], b[4];
#pragma unroll
            for (int mi = 0; mi < 2; mi++) a[mi] = as[(wm * 16 + mi * 8 + g) * SA + k];
#pragma unroll
            for (int ni = 0; ni < 4; ni++) b[ni] = bs[k * SB + wn * 32 + ni * 8 + g];
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
        }
    }
    cp_async_wait_group<0>();
#pragma unroll
    for (int mi = 0; mi < 2; mi++) {
        const int r = r0 + wm * 16 + mi * 8 + g;
        if (r >= n) continue;
#pragma unroll
        for (int ni = 0; ni < 4; ni++) {
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int b = b0 + wn * 32 + ni * 8 + 2 * t4 + i;
                if (b >= p) continue;
                double v = alpha * acc[mi][ni][i];
                if (Cin && beta != 0.0) v += beta * Cin[(size_t)r * p + b];
                Out[(size_t)r * p + b] = v;
            }
        }
    }
}

// Partial Gram tile (a0.., b0..) of A_j^T B over one chunk of rows; chunks grouped in clusters
// of 8 CTAs whose partial tiles are summed through distributed shared memory (one partial per
// cluster goes to global memory).  A gated-off CTA runs no row stages and stores nothing but
// stays for the cluster sum (see gram_dmma_cl_kernel).
__global__ void __launch_bounds__(256)
gram_pipe_kernel(int n, int p, int nb, const double *__restrict__ A, size_t strideA,
                 const double *__restrict__ B, double *__restrict__ partial, int rows_per_chunk,
                 const SolveState *st, const int *gate, const int *gate2, GramEpilogue ep) {
    const bool off = cta_gate_off(st, gate, gate2);
    namespace cg = cooperative_groups;
    constexpr int GT = 64, RS = 32, SB = GT + 4, ST = kPipeStages;
    extern __shared__ __align__(16) double psm[];
    double *As = psm;                          // ST x RS x SB
    double *Bs = psm + ST * RS * SB;           // ST x RS x SB
    const int chunk = blockIdx.x, j = blockIdx.y;
    const int ntile = (p + GT - 1) / GT;
    const int a0 = (blockIdx.z / ntile) * GT, b0 = (blockIdx.z % ntile) * GT;
    const int r_begin = chunk * rows_per_chunk;
    const int r_end = off ? r_begin : min(n, r_begin + rows_per_chunk);
    const int nst = r_end > r_begin ? (r_end - r_begin + RS - 1) / RS : 0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t4 = lane & 3;
    const double *Aj = A + (size_t)j * strideA;
    auto load = [&](int sidx, int stage) {
        const int rb = r_begin + sidx * RS;
        double *as = As + stage * RS * SB;
        double *bs = Bs + stage * RS * SB;
#pragma unroll
        for (int q = 0; q < RS * GT / 2 / 256; q++) {
            const int e = tid + q * 256;
            const int rr = e / (GT / 2), cc = (e % (GT / 2)) * 2;
            const int r = rb + rr;
            const bool rok = r < r_end;
            const bool oka = rok && a0 + cc < p, okb = rok && b0 + cc < p;
            cp_async16_zfill(as + rr * SB + cc, oka ? Aj + (size_t)r * p + a0 + cc : Aj, oka ? 16 : 0);
            cp_async16_zfill(bs + rr * SB + cc, okb ? B + (size_t)r * p + b0 + cc : B, okb ? 16 : 0);
        }
    };
    double acc[2][4][2];
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
#pragma unroll
    for (int s0 = 0; s0 < ST - 1; s0++) {
        if (s0 < nst) load(s0, s0);
        cp_async_commit_group();
    }
    for (int sidx = 0; sidx < nst; sidx++) {
        cp_async_wait_group<ST - 2>();
        __syncthreads();
        const int nxt = sidx + ST - 1;
        if (nxt < nst) load(nxt, nxt % ST);
        cp_async_commit_group();
        const double *as = As + (sidx % ST) * RS * SB;
        const double *bs = Bs + (sidx % ST) * RS * SB;
#pragma unroll
        for (int ks = 0; ks < RS / 4; ks++) {
            const int k = ks * 4 + t4;
            double a[2], b[4];
#pragma unroll
            for (int mi = 0; mi < 2; mi++) a[mi] = as[k * SB + wm * 16 + mi * 8 + g];
#pragma unroll
            for (int ni = 0; ni < 4; ni++) b[ni] = bs[k * SB + wn * 32 + ni * 8 + g];
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++) dmma884(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
        }
    }
    cp_async_wait_group<0>();
    __syncthreads();
    // this CTA's tile into its shared memory (GT x GT, row-major), then the cluster sum
    double *tile = psm;
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++)
#pragma unroll
            for (int i = 0; i < 2; i++)
                tile[(wm * 16 + mi * 8 + g) * GT + wn * 32 + ni * 8 + 2 * t4 + i] = acc[mi][ni][i];
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    const int cs = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int rpr = GT / cs;   // tile rows summed by each CTA of the cluster
    const size_t pp = (size_t)p * p;
    double *out = partial + ((size_t)(chunk / cs) * nb + j) * pp;
    for (int e = tid; e < rpr * GT; e += 256) {
        const int a = rank * rpr + e / GT, b = e % GT;
        double sum = 0.0;
        for (int q = 0; q < cs; q++) sum += cluster.map_shared_rank(tile, q)[a * GT + b];
        if (!off && a0 + a < p && b0 + b < p) {
            const size_t idx = (size_t)(a0 + a) * p + b0 + b;
            if (ep.direct) {   // one cluster per block: the final result, as the reduce kernel
                double v = ep.alpha * sum;
                if (ep.out2) ep.out2[(size_t)j * pp + idx] = v;
                if (ep.accumulate) v += ep.out[(size_t)j * pp + idx];
                ep.out[(size_t)j * pp + idx] = v;
            } else {
                out[idx] = sum;
            }
        }
    }
    cluster.sync();
}

// True when the pipelined kernels apply: 16-byte aligned rows (p even, aligned bases and
// strides) and 64-wide tiles.
static bool pipe_ok(int p, const void *A, size_t strideA, const void *B, size_t strideB) {
    if (p <= 32 || (p & 1)) return false;
    if (((uintptr_t)A | (uintptr_t)B) & 15) return false;
    if ((strideA | strideB) & 1) return false;
    return true;
}
constexpr size_t kTsmmPipeSmem = sizeof(double) * kPipeStages * (64 * 36 + 32 * 68);
constexpr size_t kGramPipeSmem = sizeof(double) * kPipeStages * 2 * 32 * 68;
extern const size_t kGramPipeSmemBytes = kGramPipeSmem;

// ---------------------------------------------------------------------------------------
// tsmm
// ---------------------------------------------------------------------------------------
template <int GT>
__global__ void __launch_bounds__(256)
tsmm_kernel(int n, int p, int nb, const double *__restrict__ A, size_t strideA,
            const double *__restrict__ S, size_t strideS, double alpha, const double *Cin,
            double beta, double *Out, const SolveState *st, const int *nb_dev, const int *gate,
            const int *gate2) {
    if (cta_gate_off(st, gate, gate2)) return;
    constexpr int TPD = GT / 16;
    constexpr int RPT = kTsmmRows / 16;
    __shared__ double As[kTsmmRows][kTsmmK + 1];
    __shared__ double Ss[kTsmmK][GT];
    const int r0 = blockIdx.x * kTsmmRows;
    const int b0 = blockIdx.y * GT;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    int nbl = nb;
    if (nb_dev) nbl = min(nb, *nb_dev);
    double acc[RPT][TPD];
#pragma unroll
    for (int i = 0; i < RPT; i++)
#pragma unroll
        for (int k = 0; k < TPD; k++) acc[i][k] = 0.0;
    for (int j = 0; j < nbl; j++) {
        const double *Aj = A + (size_t)j * strideA;
        const double *Sj = S + (size_t)j * strideS;
        for (int k0 = 0; k0 < p; k0 += kTsmmK) {
            for (int e = threadIdx.x; e < kTsmmRows * kTsmmK; e += 256) {
                const int rr = e / kTsmmK, kk = e % kTsmmK;
                const int r = r0 + rr, c = k0 + kk;
                As[rr][kk] = (r < n && c < p) ? __ldg(Aj + (size_t)r * p + c) : 0.0;
            }
            for (int e = threadIdx.x; e < kTsmmK * GT; e += 256) {
                const int kk = e / GT, cc = e % GT;
                const int a = k0 + kk, b = b0 + cc;
                Ss[kk][cc] = (a < p && b < p) ? __ldg(Sj + (size_t)a * p + b) : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < kTsmmK; kk++) {
                double a[RPT], b[TPD];
#pragma unroll
                for (int i = 0; i < RPT; i++) a[i] = As[ty + 16 * i][kk];
#pragma unroll
                for (int k = 0; k < TPD; k++) b[k] = Ss[kk][tx + 16 * k];
#pragma unroll
                for (int i = 0; i < RPT; i++)
#pragma unroll
                    for (int k = 0; k < TPD; k++) acc[i][k] = fma(a[i], b[k], acc[i][k]);
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int i = 0; i < RPT; i++) {
        const int r = r0 + ty + 16 * i;
        if (r >= n) continue;
#pragma unroll
        for (int k = 0; k < TPD; k++) {
            const int b = b0 + tx + 16 * k;
            if (b >= p) continue;
            double v = alpha * acc[i][k];
            if (Cin && beta != 0.0) v += beta * Cin[(size_t)r * p + b];
            Out[(size_t)r * p + b] = v;
        }
    }
}

bpf_status tsmm(bpf_ctx *ctx, int n, int p, int nb, const double *A, size_t strideA,
                const double *S, size_t strideS, double alpha, const double *Cin, double beta,
                double *Out, const SolveState *st, const int *nb_dev, const int *qr_gate,
                const int *gate2) {
    if (n <= 0 || p <= 0) return BPF_SUCCESS;
    const int GT = p <= 16 ? 16 : (p <= 32 ? 32 : 64);
    dim3 grid(ceil_div(n, kTsmmRows), ceil_div(p, GT));
    KScope ks(ctx, BPF_KC_TSMM, 8.0 * n * p * (nb + 1 + ((Cin && beta != 0.0) ? 1 : 0)),
              2.0 * n * p * (double)p * nb, qr_gate != nullptr || gate2 != nullptr || nb_dev != nullptr);
    if (ctx->fp64_mma && GT == 64 && !nb_dev && pipe_ok(p, A, strideA, S, strideS)) {
        BPF_CUDA(ctx, cudaFuncSetAttribute(tsmm_pipe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kTsmmPipeSmem));
        tsmm_pipe_kernel<<<grid, 256, kTsmmPipeSmem, ctx->stream>>>(n, p, nb, A, strideA, S, strideS, alpha,
                                                                    Cin, beta, Out, st, qr_gate, gate2);
    } else if (ctx->fp64_mma) {
        if (GT == 16)
            tsmm_dmma_kernel<16><<<grid, 128, 0, ctx->stream>>>(n, p, nb, A, strideA, S, strideS, alpha,
                                                                 Cin, beta, Out, st, nb_dev, qr_gate, gate2);
        else if (GT == 32)
            tsmm_dmma_kernel<32><<<grid, 128, 0, ctx->stream>>>(n, p, nb, A, strideA, S, strideS, alpha,
                                                                 Cin, beta, Out, st, nb_dev, qr_gate, gate2);
        else
            tsmm_dmma_kernel<64><<<grid, 128, 0, ctx->stream>>>(n, p, nb, A, strideA, S, strideS, alpha,
                                                                 Cin, beta, Out, st, nb_dev, qr_gate, gate2);
    } else if (GT == 16)
        tsmm_kernel<16><<<grid, 256, 0, ctx->stream>>>(n, p, nb, A, strideA, S, strideS, alpha, Cin,
                                                        beta, Out, st, nb_dev, qr_gate, gate2);
    else if (GT == 32)
        tsmm_kernel<32><<<grid, 256, 0, ctx->stream>>>(n, p, nb, A, strideA, S, strideS, alpha, Cin,
                                                        beta, Out, st, nb_dev, qr_gate, gate2);
    else
        tsmm_kernel<64><<<grid, 256, 0, ctx->stream>>>(n, p, nb, A, strideA, S, strideS, alpha, Cin,
                                                        beta, Out, st, nb_dev, qr_gate, gate2);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

__global__ void gated_copy_kernel(size_t len, const double *__restrict__ src,
                                  double *__restrict__ dst, const SolveState *st, const int *gate,
                                  const int *gate2) {
    if (cta_gate_off(st, gate, gate2)) return;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len;
         e += (size_t)gridDim.x * blockDim.x)
        dst[e] = src[e];
}

bpf_status cholqr(bpf_ctx *ctx, int n, int p, const double *W, double *Q, double *R,
                  double *T, SolveState *st, const int *gate, int *shift_flag, int *reorth_flag,
                  int iter_tag) {
    if (p > 128) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "Cholesky-QR: p=%d > 128", p);
    bpf_status s;
    double *small = (double *)ws_get(ctx, WS_SMALL, sizeof(double) * 4 * p * p, &s);
    if (!small) return s;
    double *G = small, *Rinv = small + p * p, *Rtmp = small + 2 * p * p;   // Rtmp: 2 p x p
    if (!shift_flag) shift_flag = &st->qr_shift;
    const int *g3 = shift_flag;
    // pass 1: W -> T
    BPF_TRY(gram(ctx, n, p, 1, W, 0, W, G, 1.0, false, st, gate));
    BPF_TRY(launch_chol(ctx, n, p, G, Rinv, R, Rtmp, 0, st, gate, nullptr, shift_flag, reorth_flag, iter_tag));
    BPF_TRY(tsmm(ctx, n, p, 1, W, 0, Rinv, 0, 1.0, nullptr, 0.0, T, st, nullptr, gate));
    // pass 2: T -> Q
    BPF_TRY(gram(ctx, n, p, 1, T, 0, T, G, 1.0, false, st, gate));
    BPF_TRY(launch_chol(ctx, n, p, G, Rinv, R, Rtmp, 1, st, gate, nullptr, shift_flag, nullptr, iter_tag));
    BPF_TRY(tsmm(ctx, n, p, 1, T, 0, Rinv, 0, 1.0, nullptr, 0.0, Q, st, nullptr, gate));
    // pass 3 (only when a pass needed the shift): Q -> T -> Q
    BPF_TRY(gram(ctx, n, p, 1, Q, 0, Q, G, 1.0, false, st, gate, nullptr, g3));
    BPF_TRY(launch_chol(ctx, n, p, G, Rinv, R, Rtmp, 2, st, gate, g3, nullptr, nullptr, iter_tag));
    BPF_TRY(tsmm(ctx, n, p, 1, Q, 0, Rinv, 0, 1.0, nullptr, 0.0, T, st, nullptr, gate, g3));
    size_t len = (size_t)n * p;
    int blocks = std::max(1, std::min(ceil_div((long long)len, 256), ctx->num_sms * 8));
    gated_copy_kernel<<<blocks, 256, 0, ctx->stream>>>(len, T, Q, st, gate, g3);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// Psi_i += Phi_i R1 for i < nb; C = C2 R1.  All matrices p x p row-major, R1/C2 upper.
__global__ void reorth_fold_kernel(int p, int nb, double *__restrict__ Psi,
                                   const double *__restrict__ Phi, const double *__restrict__ R1,
                                   const double *__restrict__ C2, double *__restrict__ C,
                                   double *__restrict__ scratch, const SolveState *st,
                                   const int *gate) {
    if (cta_gate_off(st, gate)) return;
    const size_t pp = (size_t)p * p;
    const size_t total = (size_t)nb * pp;
    // blocks 0..nb-1: Psi update; block nb (one extra p x p) : C2 R1 into scratch
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total + pp; e += stride) {
        if (e < total) {
            const size_t blk = e / pp;
            const int a = (int)((e % pp) / p), b = (int)(e % p);
            const double *ph = Phi + blk * pp + (size_t)a * p;
            double s = 0.0;
            for (int c = 0; c <= b; c++) s += ph[c] * R1[(size_t)c * p + b];
            Psi[e] += s;
        } else {
            const size_t f = e - total;
            const int a = (int)(f / p), b = (int)(f % p);
            double s = 0.0;
            for (int c = a; c <= b; c++) s += C2[(size_t)a * p + c] * R1[(size_t)c * p + b];
            scratch[f] = (b >= a) ? s : 0.0;
        }
    }
}

bpf_status reorth_fold(bpf_ctx *ctx, int p, int nb, double *Psi, const double *Phi,
                       const double *R1, const double *C2, double *C, double *scratch,
                       const SolveState *st, const int *gate) {
    const size_t work = (size_t)(nb + 1) * p * p;
    int blocks = std::max(1, std::min(ceil_div((long long)work, 256), ctx->num_sms * 4));
    reorth_fold_kernel<<<blocks, 256, 0, ctx->stream>>>(p, nb, Psi, Phi, R1, C2, C, scratch, st, gate);
    BPF_LAUNCHED(ctx);
    const size_t pp = (size_t)p * p;
    blocks = std::max(1, std::min(ceil_div((long long)pp, 256), ctx->num_sms));
    gated_copy_kernel<<<blocks, 256, 0, ctx->stream>>>(pp, scratch, C, st, gate, nullptr);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// ---------------------------------------------------------------------------------------
// elementwise and reductions
// ---------------------------------------------------------------------------------------
__global__ void axpby_kernel(size_t len, double a, const double *__restrict__ x, double b,
                             double *__restrict__ y, const SolveState *st) {
    if (cta_gate_off(st, nullptr)) return;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len;
         e += (size_t)gridDim.x * blockDim.x)
        y[e] = a * x[e] + (b == 0.0 ? 0.0 : b * y[e]);
}

bpf_status axpby(bpf_ctx *ctx, size_t len, double a, const double *x, double b, double *y,
                 const SolveState *st) {
    if (len == 0) return BPF_SUCCESS;
    int blocks = std::max(1, std::min(ceil_div((long long)len, 256), ctx->num_sms * 8));
    axpby_kernel<<<blocks, 256, 0, ctx->stream>>>(len, a, x, b, y, st);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

// Deterministic two-stage sum of squares: stage 1 one partial per block, stage 2 one block.
__global__ void sumsq_partial_kernel(size_t len, const double *__restrict__ x,
                                     double *__restrict__ part) {
    double s = 0.0;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len;
         e += (size_t)gridDim.x * blockDim.x)
        s += x[e] * x[e];
    s = warp_sum(s);
    __shared__ double ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) part[blockIdx.x] = v;
    }
}

__global__ void sum_sqrt_kernel(int nparts, const double *__restrict__ part, double *out) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
    s = warp_sum(s);
    __shared__ double ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) *out = sqrt(v);
    }
}

bpf_status frob_norm(bpf_ctx *ctx, size_t len, const double *x, double *out) {
    bpf_status s;
    const int nparts = ctx->num_sms * 2;
    double *buf = (double *)ws_get(ctx, WS_NORM, sizeof(double) * nparts, &s);
    if (!buf) return s;
    sumsq_partial_kernel<<<nparts, 256, 0, ctx->stream>>>(len, x, buf);
    BPF_LAUNCHED(ctx);
    sum_sqrt_kernel<<<1, 256, 0, ctx->stream>>>(nparts, buf, out);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

}  // namespace bpf

// ---------------------------------------------------------------------------------------
// C ABI: householder!(Q, R) on a column-major block (src/block_utils.jl:46-53)
// ---------------------------------------------------------------------------------------
using namespace bpf;

namespace bpf {

// Householder vectors of an orthonormal Q (row-major n x p, positive-diagonal R from Cholesky-QR)
// in LAPACK's geqrf form, by reconstruction (Ballard et al., "Reconstructing Householder vectors
// from tall-skinny QR", 2015): the LU without pivoting of Q - [S; 0], where the sign s_j is taken
// opposite to the running pivot, gives the unit lower trapezoidal Y = [Y1; Y2] of the reflectors
// and U = -T Y1^T S, so tau_j = T_jj = -U_jj s_j; Q S is what orgqr returns and S R its R (the
// R of Householder QR applied to the original block, with LAPACK's signs).  One CTA: the p x p
// top block is factored in shared memory (s_j, tau_j, strict lower L1 = Y1), U^{-1} is formed by
// column-wise back substitution (a thread per column) for Y2 = Q2 U^{-1}.
__global__ void house_recon_kernel(int p, const double *__restrict__ Qtop, const double *__restrict__ R,
                                   double *__restrict__ sgn, double *__restrict__ tau,
                                   double *__restrict__ Uinv, double *__restrict__ Ctop) {
    extern __shared__ double M[];   // p x p, row-major
    __shared__ double s_piv;
    for (int idx = threadIdx.x; idx < p * p; idx += blockDim.x) M[idx] = Qtop[idx];
    __syncthreads();
    for (int j = 0; j < p; j++) {
        if (threadIdx.x == 0) {
            const double a = M[j * p + j];
            const double s = a >= 0.0 ? -1.0 : 1.0;   // LAPACK: beta = -sign(alpha) ||x||
            sgn[j] = s;
            M[j * p + j] = a - s;                      // |a - s| >= 1
            s_piv = a - s;
        }
        __syncthreads();
        const double piv = s_piv;
        for (int i = j + 1 + threadIdx.x; i < p; i += blockDim.x) M[i * p + j] /= piv;
        __syncthreads();
        const int rows = p - j - 1;
        for (int idx = threadIdx.x; idx < rows * rows; idx += blockDim.x) {
            const int i = j + 1 + idx / rows, k = j + 1 + idx % rows;
            M[i * p + k] -= M[i * p + j] * M[j * p + k];
        }
        __syncthreads();
    }
    // tau, the compact top block (upper: S R; strict lower: L1) and U^{-1}
    for (int idx = threadIdx.x; idx < p * p; idx += blockDim.x) {
        const int i = idx / p, k = idx % p;
        Ctop[idx] = k >= i ? sgn[i] * R[idx] : M[idx];
    }
    for (int j = threadIdx.x; j < p; j += blockDim.x) tau[j] = -M[j * p + j] * sgn[j];
    for (int k = threadIdx.x; k < p; k += blockDim.x) {
        for (int i = p - 1; i >= 0; i--) {
            if (i > k) {
                Uinv[i * p + k] = 0.0;
                continue;
            }
            double v = (i == k) ? 1.0 : 0.0;
            for (int l = i + 1; l <= k; l++) v -= M[i * p + l] * Uinv[l * p + k];
            Uinv[i * p + k] = v / M[i * p + i];
        }
    }
}

// Columns of a row-major n x p block scaled by s (Q S), rows of a p x p matrix (S R).
__global__ void scale_cols_kernel(size_t n, int p, const double *__restrict__ s, double *__restrict__ X) {
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n * p; idx += (size_t)gridDim.x * blockDim.x)
        X[idx] *= s[idx % p];
}
__global__ void scale_rows_kernel(int p, const double *__restrict__ s, double *__restrict__ R) {
    for (int idx = threadIdx.x; idx < p * p; idx += blockDim.x) R[idx] *= s[idx / p];
}

}  // namespace bpf

extern "C" bpf_status bpf_householder_lapack(bpf_ctx *ctx, int n, int p, double *Q, int ldq, double *R,
                                             int ldr, double *tau, int compact) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    if (n < 0 || p < 0 || (n > 0 && p > 0 && (!Q || !R)))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "householder: invalid argument");
    if (ldq < std::max(1, n) || ldr < std::max(1, p))
        return set_error(ctx, BPF_ERR_DIMENSION, "householder: leading dimension too small");
    if (p > n) return set_error(ctx, BPF_ERR_DIMENSION, "householder: n=%d < p=%d", n, p);
    if (n == 0 || p == 0) return BPF_SUCCESS;
    if (p > 128) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "householder: p=%d > 128", p);
    const size_t np = (size_t)n * p, pp = (size_t)p * p;
    bpf_status s;
    double *buf = (double *)ws_get(ctx, WS_A, sizeof(double) * (3 * np + 4 * pp + 2 * (size_t)p), &s);
    if (!buf) return s;
    double *W = buf, *Qr = buf + np, *T = buf + 2 * np, *Rr = buf + 3 * np, *Uinv = Rr + pp, *Ctop = Uinv + pp,
           *Rl = Ctop + pp, *sg = Rl + pp, *tau_d = sg + p;
    SolveState *st = (SolveState *)ws_get(ctx, WS_STATE, sizeof(SolveState), &s);
    if (!st) return s;
    SolveState hs;
    memset(&hs, 0, sizeof(hs));
    hs.active = 1;
    BPF_CUDA(ctx, cudaMemcpyAsync(st, &hs, sizeof(SolveState), cudaMemcpyHostToDevice, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    BPF_TRY(colmajor_to_rowmajor(ctx, n, p, Q, ldq, W));
    BPF_TRY(cholqr(ctx, n, p, W, Qr, Rr, T, st));
    const size_t smem = sizeof(double) * pp;
    BPF_CUDA(ctx, cudaFuncSetAttribute(house_recon_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    house_recon_kernel<<<1, 256, smem, ctx->stream>>>(p, Qr, Rr, sg, tau_d, Uinv, Ctop);
    BPF_LAUNCHED(ctx);
    BPF_CUDA(ctx, cudaMemcpyAsync(Rl, Rr, sizeof(double) * pp, cudaMemcpyDeviceToDevice, ctx->stream));
    scale_rows_kernel<<<1, 256, 0, ctx->stream>>>(p, sg, Rl);
    BPF_LAUNCHED(ctx);
    if (compact) {
        // [Ctop; Q2 U^{-1}] in W (row-major), then to the caller's column-major Q
        BPF_CUDA(ctx, cudaMemcpyAsync(W, Ctop, sizeof(double) * pp, cudaMemcpyDeviceToDevice, ctx->stream));
        if (n > p) BPF_TRY(tsmm(ctx, n - p, p, 1, Qr + pp, 0, Uinv, 0, 1.0, nullptr, 0.0, W + pp, st));
        BPF_TRY(rowmajor_to_colmajor(ctx, n, p, W, Q, ldq));
    } else {
        const int g = (int)std::max<long long>(1, std::min<long long>(ceil_div((long long)np, 256LL), 4LL * ctx->num_sms));
        scale_cols_kernel<<<g, 256, 0, ctx->stream>>>(n, p, sg, Qr);
        BPF_LAUNCHED(ctx);
        BPF_TRY(rowmajor_to_colmajor(ctx, n, p, Qr, Q, ldq));
    }
    BPF_TRY(rowmajor_to_colmajor(ctx, p, p, Rl, R, ldr));
    if (tau) BPF_CUDA(ctx, cudaMemcpyAsync(tau, tau_d, sizeof(double) * p, cudaMemcpyDeviceToDevice, ctx->stream));
    return check_dev_status(ctx, "householder");
}

extern "C" bpf_status bpf_householder(bpf_ctx *ctx, int n, int p, double *Q, int ldq, double *R,
                                      int ldr) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    if (n < 0 || p < 0 || (n > 0 && p > 0 && (!Q || !R)))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "householder: invalid argument");
    if (ldq < std::max(1, n) || ldr < std::max(1, p))
        return set_error(ctx, BPF_ERR_DIMENSION, "householder: leading dimension too small");
    if (p > n) return set_error(ctx, BPF_ERR_DIMENSION, "householder: n=%d < p=%d", n, p);
    if (n == 0 || p == 0) return BPF_SUCCESS;
    if (p > 128) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "householder: p=%d > 128", p);
    const size_t np = (size_t)n * p, pp = (size_t)p * p;
    bpf_status s;
    double *buf = (double *)ws_get(ctx, WS_A, sizeof(double) * (3 * np + 2 * pp), &s);
    if (!buf) return s;
    double *W = buf, *Qr = buf + np, *T = buf + 2 * np, *Rr = buf + 3 * np;
    SolveState *st = (SolveState *)ws_get(ctx, WS_STATE, sizeof(SolveState), &s);
    if (!st) return s;
    SolveState hs;
    memset(&hs, 0, sizeof(hs));
    hs.active = 1;
    BPF_CUDA(ctx, cudaMemcpyAsync(st, &hs, sizeof(SolveState), cudaMemcpyHostToDevice, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    BPF_TRY(colmajor_to_rowmajor(ctx, n, p, Q, ldq, W));
    BPF_TRY(cholqr(ctx, n, p, W, Qr, Rr, T, st));
    BPF_TRY(rowmajor_to_colmajor(ctx, n, p, Qr, Q, ldq));
    BPF_TRY(rowmajor_to_colmajor(ctx, p, p, Rr, R, ldr));
    return check_dev_status(ctx, "householder");
}
