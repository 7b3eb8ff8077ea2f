// Block-Jacobi preconditioner: the inverses of the diagonal blocks of A, applied by
// multiplication (mul! semantics).
//
// Reference: the reference's tests and benchmark use ExaPF's LinearSolvers.BlockJacobi-
// Preconditioner (ExaPF 0.9.3, an external package not vendored with the reference):
// test/block_gmres.jl:5,17,22 and benchmarks/benchmarks_nvidia.jl:47-51 build it with
// div(n, 32) blocks and pass it to block_gmres as N with ldiv = false, i.e. y = P x with P the
// block-diagonal matrix of the blocks' dense inverses.  ExaPF partitions the rows with METIS; no
// METIS library is available here, so the blocks are consecutive runs of `block_size` rows in a
// chosen order (natural, or reverse Cuthill-McKee / minimum degree to keep coupled rows
// together).  The inverse of every block is dense and exact (Gauss-Jordan with partial pivoting).
//
// Design (B200): one warp per block for the set-up (the block gathered from the CSR rows into
// shared memory as [A_b | I], Gauss-Jordan on it, lanes over the 64 columns), one warp per
// (block, 32-column slice) for the apply (the block's rows of X staged in shared memory, the
// 32 x 32 inverse read through L1).  In-place application is safe: a warp reads all of its rows
// before it writes them, and warps of one block own disjoint columns.
#include <algorithm>
#include <numeric>
#include <vector>

#include "bpf_internal.cuh"
#include "ordering.cuh"
#include "prec.cuh"

namespace bpf {

constexpr int kBJ = 32;   // largest block (rows); blocks are stored padded to kBJ x kBJ

__global__ void __launch_bounds__(64) bj_setup_kernel(int nblk, const int *__restrict__ rows,
                                                      const int *__restrict__ rp, const int *__restrict__ ci,
                                                      const double *__restrict__ av, const int *__restrict__ blk_of,
                                                      const int *__restrict__ loc, double *__restrict__ inv,
                                                      DevStatus *ds) {
    __shared__ double Ms[2][kBJ][2 * kBJ + 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int b = blockIdx.x * 2 + w;
    if (b >= nblk) return;   // warp-uniform; no CTA barrier below
    double(*M)[2 * kBJ + 1] = Ms[w];
    const int *rb = rows + (size_t)b * kBJ;
    int sz = 0;
    for (int i = 0; i < kBJ; i++) sz += rb[i] >= 0 ? 1 : 0;
    for (int i = 0; i < kBJ; i++) {
        M[i][lane] = 0.0;
        M[i][kBJ + lane] = i == lane ? 1.0 : 0.0;
    }
    __syncwarp();
    if (lane < sz) {   // lane = local row
        const int r = rb[lane];
        for (int k = rp[r]; k < rp[r + 1]; k++) {
            const int c = ci[k];
            if (blk_of[c] == b) M[lane][loc[c]] = av[k];
        }
    }
    __syncwarp();
    int singular = 0;
    for (int k = 0; k < sz; k++) {
        // pivot: the largest |M[i][k]| over i >= k (smallest i on ties)
        double v = (lane >= k && lane < sz) ? fabs(M[lane][k]) : -1.0;
        int idx = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
            const int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
            if (v2 > v || (v2 == v && i2 < idx)) {
                v = v2;
                idx = i2;
            }
        }
        if (!(v > 0.0)) {
            singular = 1;
            break;
        }
        if (idx != k) {
            const double a0 = M[k][lane], a1 = M[k][kBJ + lane];
            M[k][lane] = M[idx][lane];
            M[k][kBJ + lane] = M[idx][kBJ + lane];
            M[idx][lane] = a0;
            M[idx][kBJ + lane] = a1;
        }
        __syncwarp();
        const double d = 1.0 / M[k][k];
        __syncwarp();
        M[k][lane] *= d;
        M[k][kBJ + lane] *= d;
        __syncwarp();
        for (int i = 0; i < sz; i++) {
            if (i == k) continue;
            const double f = M[i][k];
            __syncwarp();
            M[i][lane] -= f * M[k][lane];
            M[i][kBJ + lane] -= f * M[k][kBJ + lane];
            __syncwarp();
        }
    }
    if (singular) {
        if (lane == 0 && atomicCAS(&ds->err, 0, (int)DEV_ZERO_PIVOT) == 0) ds->aux = b;
        return;
    }
    double *ib = inv + (size_t)b * kBJ * kBJ;
    for (int i = 0; i < kBJ; i++) ib[i * kBJ + lane] = (i < sz && lane < sz) ? M[i][kBJ + lane] : 0.0;
}

// Y (row-major n x p) = P X, P = diag(inv_b); Y may be X.
__global__ void __launch_bounds__(128) bj_apply_kernel(int nblk, int p, const int *__restrict__ rows,
                                                       const double *__restrict__ inv, const double *X,
                                                       double *Y) {
    __shared__ double Xs[4][kBJ][kBJ + 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nchunk = (p + 31) / 32;
    const long long task = (long long)blockIdx.x * 4 + w;
    const int b = (int)(task / nchunk);
    if (b >= nblk) return;
    const int col = (int)(task % nchunk) * 32 + lane;
    const int *rb = rows + (size_t)b * kBJ;
    int sz = 0;
    for (int i = 0; i < kBJ; i++) {
        const int r = rb[i];
        sz += r >= 0 ? 1 : 0;
        Xs[w][i][lane] = (r >= 0 && col < p) ? X[(size_t)r * p + col] : 0.0;
    }
    __syncwarp();
    const double *ib = inv + (size_t)b * kBJ * kBJ;
    for (int i = 0; i < sz; i++) {
        double acc = 0.0;
#pragma unroll 8
        for (int j = 0; j < kBJ; j++) acc += __ldg(ib + i * kBJ + j) * Xs[w][j][lane];
        if (col < p) Y[(size_t)rb[i] * p + col] = acc;
    }
}

bpf_status bj_setup(bpf_ctx *ctx, bpf_prec *P) {
    if (P->bj_nblk == 0) return BPF_SUCCESS;
    const int grid = ceil_div(P->bj_nblk, 2);
    KScope ks(ctx, BPF_KC_FACTOR, 12.0 * P->nnz + 8.0 * P->bj_nblk * kBJ * kBJ, 0.0);
    bj_setup_kernel<<<grid, 64, 0, ctx->stream>>>(P->bj_nblk, P->bj_rows, P->rp, P->ci, P->fv, P->bj_blk,
                                                  P->bj_loc, P->bj_inv, ctx->dstat);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

bpf_status bj_apply_rowmajor(bpf_ctx *ctx, const bpf_prec *P, int p, const double *X, double *Y) {
    if (P->bj_nblk == 0 || p == 0) return BPF_SUCCESS;
    const long long tasks = (long long)P->bj_nblk * ((p + 31) / 32);
    const int grid = (int)((tasks + 3) / 4);
    KScope ks(ctx, BPF_KC_TRSV, 8.0 * P->bj_nblk * kBJ * kBJ + 16.0 * P->n * p, 2.0 * P->bj_nblk * kBJ * kBJ * (double)p);
    bj_apply_kernel<<<grid, 128, 0, ctx->stream>>>(P->bj_nblk, p, P->bj_rows, P->bj_inv, X, Y);
    BPF_LAUNCHED(ctx);
    return BPF_SUCCESS;
}

}  // namespace bpf

using namespace bpf;

extern "C" bpf_status bpf_block_jacobi_create(bpf_ctx *ctx, const bpf_csr_desc *A, int block_size, int ordering,
                                              bpf_prec **out) {
    if (!ctx || !out) return BPF_ERR_INVALID_VALUE;
    *out = nullptr;
    if (!A) return set_error(ctx, BPF_ERR_INVALID_VALUE, "null matrix");
    if (A->dtype != BPF_F64) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "FP64 matrices only");
    if (block_size < 1 || block_size > kBJ)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "block-Jacobi: block size must be 1..%d", kBJ);
    if (ordering == BPF_ORDER_METIS)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "block-Jacobi: a METIS partition needs a METIS library");
    if (ordering < 0 || ordering > BPF_ORDER_NATURAL)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "unknown ordering %d", ordering);
    std::vector<int> rp, ci;
    BPF_TRY(csr_pattern_to_host(ctx, A, rp, ci, false, nullptr));
    const int n = A->n, nnz = A->nnz;
    std::vector<int> order(n);
    if (ordering == BPF_ORDER_NATURAL) std::iota(order.begin(), order.end(), 0);
    else if (ordering == BPF_ORDER_RCM) order = order_rcm(n, rp, ci);
    else order = order_min_degree(n, rp, ci);
    const int nblk = (n + block_size - 1) / block_size;
    std::vector<int> rows((size_t)nblk * kBJ, -1), blk(n), loc(n);
    for (int k = 0; k < n; k++) {
        const int b = k / block_size, i = k % block_size;
        rows[(size_t)b * kBJ + i] = order[k];
        blk[order[k]] = b;
        loc[order[k]] = i;
    }
    bpf_prec *P = new bpf_prec();
    P->ctx = ctx;
    P->kind = PREC_BJ;
    P->n = n;
    P->nnz = nnz;
    P->nrhs = 1;
    P->ordering = ordering;
    P->bj_nblk = nblk;
    P->bj_bs = block_size;
    P->perm_host = order;   // the row order the blocks are cut from (bpf_prec_permutation)
    auto fail = [&](bpf_status s) {
        bpf_prec_destroy(P);
        return s;
    };
    cudaError_t e = cudaSuccess;
    auto up = [&](int **d, const std::vector<int> &h) {
        if (e == cudaSuccess && !h.empty()) e = cudaMalloc((void **)d, sizeof(int) * h.size());
        if (e == cudaSuccess && !h.empty())
            e = cudaMemcpy(*d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice);
    };
    up(&P->rp, rp);
    up(&P->ci, ci);
    up(&P->bj_rows, rows);
    up(&P->bj_blk, blk);
    up(&P->bj_loc, loc);
    if (e == cudaSuccess && nnz > 0) e = cudaMalloc((void **)&P->fv, sizeof(double) * nnz);
    if (e == cudaSuccess) e = cudaMalloc((void **)&P->bj_inv, sizeof(double) * (size_t)nblk * kBJ * kBJ);
    if (e != cudaSuccess) return fail(cuda_error(ctx, e, "block-Jacobi setup", __FILE__, __LINE__));
    bpf_status s = bpf_prec_refactor(P, (const double *)A->vals);
    if (s != BPF_SUCCESS) return fail(s);
    *out = P;
    return BPF_SUCCESS;
}
