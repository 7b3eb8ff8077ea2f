// block-GMRES: src/block_gmres.jl:127-411 (block_gmres / block_gmres!).
//
// The host drives restart passes; the inner Arnoldi iterations run device-resident.  Every
// kernel of iteration k reads SolveState::active and returns at once when the device-side
// stopping test (residual <= eps, inner itmax, time limit) has ended the pass, so the host
// launches a chunk of iterations and synchronises once per chunk instead of once per
// iteration (the reference syncs on norm(C) every iteration, :342).
//
// Per iteration k (k = 1-based, j = k-1):
//   P = N \ V_j                    one cooperative ILU0/IC0 launch           (:298)
//   W = A P                        CSR SpMM                                  (:299)
//   Q = M \ W                      (left preconditioner, if any)             (:300)
//   Psi = V^T Q, Q -= V Psi  x2    block classical Gram-Schmidt, two passes  (:301-313)
//   V_{j+1} C = Q                  Cholesky-QR2 (shifted on breakdown)        (:316)
//   apply Omega_0..Omega_{j-1}     compact-WY block reflectors, p CTAs        (:318-326)
//   factor [R_jj; C], update Z     one CTA; ||Lambda_{j+1}||_F -> stop test   (:328-353)
// End of a pass: block back substitution (p CTAs), X += sum V_i Y_i, X <- N X   (:366-385)
//
// Numerics vs the reference: two classical Gram-Schmidt passes instead of modified GS
// (+ optional reorthogonalization), Cholesky-QR instead of Householder for the basis blocks
// (R has a positive diagonal, LAPACK's may be negative).  Both produce the same Krylov basis
// up to column signs, so X and the residual history agree up to rounding.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "bpf_internal.cuh"
#include "dense.cuh"
#include "prec.cuh"
#include "small.cuh"

namespace bpf {


__device__ __forceinline__ double block_sum(double v, double *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double t = lane < nw ? red[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) red[0] = t;
    }
    __syncthreads();
    double r = red[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void gmres_init_kernel(SolveState *st, double atol, double rtol, double *hist,
                                  double timemax) {
    const double r = st->rnorm;
    st->eps = atol + rtol * r;
    st->solved = r <= st->eps;
    if (st->hist_cap > 0) hist[0] = r;
    st->nres = 1;
    st->active = 0;
    st->inner_iter = 0;
    st->overtimed = 0;
    st->deadline_ns = (timemax > 0.0 && timemax < 1e15) ? globaltimer_ns() + (unsigned long long)(timemax * 1e9) : 0ull;
}

__global__ void pass_begin_kernel(SolveState *st, int inner_itmax) {
    st->qr_fail_iter = 0x7fffffff;
    st->inner_itmax = inner_itmax;
    st->inner_iter = 0;
    st->inner_tired = 0;
    st->active = !(st->solved || st->overtimed);
}

// Grow a workspace slot to `bytes`, keeping its first `keep` bytes.
bpf_status ws_grow_keep(bpf_ctx *ctx, int slot, size_t bytes, size_t keep) {
    if (ctx->ws_bytes[slot] >= bytes) return BPF_SUCCESS;
    void *p = nullptr;
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    BPF_CUDA(ctx, cudaMalloc(&p, bytes));
    if (ctx->ws[slot] && keep)
        BPF_CUDA(ctx, cudaMemcpyAsync(p, ctx->ws[slot], std::min(keep, ctx->ws_bytes[slot]),
                                      cudaMemcpyDeviceToDevice, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->ws[slot]) cudaFree(ctx->ws[slot]);
    ctx->ws[slot] = p;
    ctx->ws_bytes[slot] = bytes;
    return BPF_SUCCESS;
}

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// dst (n x p, row-major) = src (n x r, row-major) in the first r columns, zeros after.
__global__ void pad_cols_kernel(int n, int r, int p, const double *__restrict__ src, double *__restrict__ dst) {
    const size_t total = (size_t)n * p;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t i = e / p;
        const int c = (int)(e % p);
        dst[e] = c < r ? src[i * r + c] : 0.0;
    }
}

// Columns c0 <= c < c1 of the row-major n x p block X set to zero.
__global__ void zero_cols_kernel(int n, int c0, int c1, int p, double *__restrict__ X) {
    const size_t total = (size_t)n * (c1 - c0);
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
        X[(e / (c1 - c0)) * p + c0 + e % (c1 - c0)] = 0.0;
}

// Deflation state of one solve (GCRO form): Q_C = A Z R^{-1} orthonormal (n x r, zero-padded
// to p columns), Zd = Z R^{-1} (so that A Zd = Q_C), E_j = Q_C^T (A N^{-1} V_j) per iteration
// and the accumulated correction Xdef of the current pass.
struct Deflation {
    int r = 0;
    double *Qp = nullptr, *Zp = nullptr, *Xdef = nullptr, *E = nullptr, *E2 = nullptr, *F = nullptr;
};

struct GmresBufs {
    double *V, *Rblk, *HY, *tau, *Z;
    double *Zb;   // flexible form: preconditioned basis N \ V_i (null otherwise)
    int cap;
};

static bpf_status gmres_capacity(bpf_ctx *ctx, int n, int p, int cap, int old_cap, GmresBufs &g,
                                 bool flexible) {
    const size_t np = (size_t)n * p, pp = (size_t)p * p;
    BPF_TRY(ws_grow_keep(ctx, WS_V, sizeof(double) * np * (cap + 1), sizeof(double) * np * (old_cap + 1)));
    if (flexible) {
        BPF_TRY(ws_grow_keep(ctx, WS_ZB, sizeof(double) * np * cap, sizeof(double) * np * old_cap));
        g.Zb = (double *)ctx->ws[WS_ZB];
    } else {
        g.Zb = nullptr;
    }
    BPF_TRY(ws_grow_keep(ctx, WS_HESS, sizeof(double) * pp * ((size_t)cap * (cap + 1) / 2),
                         sizeof(double) * pp * ((size_t)old_cap * (old_cap + 1) / 2)));
    BPF_TRY(ws_grow_keep(ctx, WS_HY, sizeof(double) * hy_stride(p) * cap,
                         sizeof(double) * hy_stride(p) * old_cap));
    BPF_TRY(ws_grow_keep(ctx, WS_Z, sizeof(double) * pp * (cap + 1), sizeof(double) * pp * (old_cap + 1)));
    g.V = (double *)ctx->ws[WS_V];
    g.Rblk = (double *)ctx->ws[WS_HESS];
    g.HY = (double *)ctx->ws[WS_HY];
    g.Z = (double *)ctx->ws[WS_Z];
    g.cap = cap;
    return BPF_SUCCESS;
}

}  // namespace bpf

using namespace bpf;

static bpf_status block_gmres_impl(bpf_ctx *ctx, const bpf_csr_desc *A, int p, const double *B,
                                   int ldb, double *X, int ldx, const double *X0, int ldx0,
                                   const bpf_prec *M, const bpf_prec *N, const bpf_gmres_opts *opts,
                                   bpf_stats *stats, const double *Zdef, int ldz, int rdef) {
    if (!ctx) return BPF_ERR_INVALID_VALUE;
    const double t0 = now_s();
    if (!A || !opts || !stats) return set_error(ctx, BPF_ERR_INVALID_VALUE, "block_gmres: null argument");
    const int n = A->n;
    if (A->dtype != BPF_F64) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "block_gmres: FP64 matrices only");
    if (n < 1 || p < 1 || !B || !X) return set_error(ctx, BPF_ERR_INVALID_VALUE, "block_gmres: empty system");
    if (ldb < n || ldx < n || (X0 && ldx0 < n))
        return set_error(ctx, BPF_ERR_DIMENSION, "Inconsistent problem size");
    if ((M && M->n != n) || (N && N->n != n))
        return set_error(ctx, BPF_ERR_DIMENSION, "preconditioner size differs from the system");
    // ILU0 / IC0 define only ldiv! (the reference's mul! is undefined for them); block-Jacobi,
    // ExaPF's preconditioner in the reference's tests, is applied by mul! (ldiv = false).
    const bool m_bj = M && M->kind == PREC_BJ, n_bj = N && N->kind == PREC_BJ;
    if (((M && !m_bj) || (N && !n_bj)) && !opts->ldiv)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED,
                         "ILU0/IC0 preconditioners define only ldiv!: pass ldiv=true");
    if ((m_bj || n_bj) && opts->ldiv)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED,
                         "block-Jacobi is applied by mul!: pass ldiv=false");
    if (p > n) return set_error(ctx, BPF_ERR_DIMENSION, "block_gmres: p=%d > n=%d", p, n);
    if (p > 128) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "block_gmres: p=%d > 128", p);
    if (rdef > 0) {
        if (!Zdef || ldz < n) return set_error(ctx, BPF_ERR_INVALID_VALUE, "block_gmres: deflation basis");
        if (rdef > p)
            return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "block_gmres: deflation rank %d > p = %d", rdef, p);
        if (M) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "block_gmres: deflation with a left preconditioner");
    }
    // reordered preconditioners: their scratch must hold p columns before the loop starts
    if (M) BPF_TRY(prec_reserve_z(ctx, const_cast<bpf_prec *>(M), p));
    if (N) BPF_TRY(prec_reserve_z(ctx, const_cast<bpf_prec *>(N), p));
    int memory = std::min(n / p, opts->memory);
    if (memory < 1) memory = 1;
    const bool restart = opts->restart != 0;
    int itmax = opts->itmax == 0 ? 2 * (n / p) : opts->itmax;
    if (itmax < 0) itmax = 0;
    const double timemax = (opts->timemax > 0.0) ? opts->timemax : 1e300;
    const size_t np = (size_t)n * p, pp = (size_t)p * p;
    bpf_status s;

    // n x p working blocks
    double *vec = (double *)ws_get(ctx, WS_VEC, sizeof(double) * np * 7, &s);
    if (!vec) return s;
    double *Bi = vec, *Xi = vec + np, *W = vec + 2 * np, *Qm = vec + 3 * np, *Pm = vec + 4 * np,
           *dX = vec + 5 * np, *Tq = vec + 6 * np;
    double *R0 = M ? Qm : W;
    double *Xr = restart ? dX : Xi;
    SolveState *st = (SolveState *)ws_get(ctx, WS_STATE, sizeof(SolveState), &s);
    if (!st) return s;
    const int hist_cap = itmax + 2;
    double *hist = (double *)ws_get(ctx, WS_HIST, sizeof(double) * hist_cap, &s);
    if (!hist) return s;
    // C blocks by iteration parity (2 p x p), C2 and fold scratch (2 p x p), tau (p), scratch of
    // the factor kernel (3 p (p+1) + p; used for p > 64 only)
    const size_t hscr_n = 4 * pp + p + 3 * (size_t)p * (p + 1) + p;
    double *hscr = (double *)ws_get(ctx, WS_HSCR, sizeof(double) * hscr_n, &s);
    if (!hscr) return s;
    double *Cpar[2] = {hscr, hscr + pp};
    double *C2 = hscr + 2 * pp;
    double *fold_scr = hscr + 3 * pp;
    double *tau_cur = hscr + 4 * pp;
    double *scr = hscr + 4 * pp + p;
    // The Hessenberg update of iteration k runs on the second stream, overlapped with the
    // Arnoldi step of iteration k+1 (it feeds only the stopping test and the next update).
    // Kernels of the main stream may then run up to two iterations past the converged one;
    // those iterations only write basis blocks and Hessenberg columns beyond the solution's.
    const bool overlap = ctx->overlap && ctx->hstream != nullptr;
    int last_hess = 0;   // iteration of the last Hessenberg update enqueued on the second stream
    auto join = [&]() -> bpf_status {   // main stream waits for the last Hessenberg update
        if (overlap && last_hess > 0)
            BPF_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_b[last_hess & 1], 0));
        return BPF_SUCCESS;
    };
    GmresBufs g{};
    // An FP32-factor right preconditioner is not exactly the same linear map at every
    // application (rounding), so the flexible form keeps the preconditioned blocks
    // Zb_i = N \ V_i and forms X += sum Zb_i Y_i (Saad's FGMRES); the Arnoldi relation
    // A Zb = V H then holds in FP64 and the residual estimate stays the true residual.
    const bool flexible = N && N->fdtype == BPF_F32;
    int cap = restart ? std::min(memory, std::max(itmax, 1)) : std::min(std::max(itmax, 1), std::max(memory, 16));
    BPF_TRY(gmres_capacity(ctx, n, p, cap, 0, g, flexible));

    // State on the host side.
    SolveState hs;
    std::memset(&hs, 0, sizeof(hs));
    hs.itmax = itmax;
    hs.active = 1;   // lets the set-up products run; gmres_init_kernel decides the first pass
    hs.qr_fail_iter = 0x7fffffff;
    hs.inner_itmax = itmax;
    hs.mem = memory;
    hs.restart = restart;
    hs.hist_cap = hist_cap;
    hs.atol = opts->atol;
    hs.rtol = opts->rtol;
    BPF_CUDA(ctx, cudaMemcpyAsync(st, &hs, sizeof(SolveState), cudaMemcpyHostToDevice, ctx->stream));

    // Initial residual (:215-227).
    const int base = A->index_base;
    const int *rp = A->rowptr, *ci = A->colind;
    const double *av = (const double *)A->vals;
    BPF_TRY(colmajor_to_rowmajor(ctx, n, p, B, ldb, Bi));
    BPF_CUDA(ctx, cudaMemsetAsync(Xi, 0, sizeof(double) * np, ctx->stream));
    const bool warm = X0 != nullptr;
    if (warm) {
        BPF_TRY(colmajor_to_rowmajor(ctx, n, p, X0, ldx0, dX));
        BPF_TRY(spmm_rowmajor(ctx, n, A->nnz, rp, ci, av, base, p, 1.0, dX, 0.0, W, Bi));
        if (restart) BPF_CUDA(ctx, cudaMemcpyAsync(Xi, dX, sizeof(double) * np, cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
        BPF_CUDA(ctx, cudaMemcpyAsync(W, Bi, sizeof(double) * np, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    if (M) BPF_TRY(prec_apply_rowmajor(ctx, M, p, W, Qm));
    BPF_TRY(frob_norm(ctx, np, R0, &st->rnorm));
    Deflation dfl;
    if (rdef > 0) {
        // Q_C = A Z R^{-1} by Cholesky-QR (R on the host for its inverse), Zd = Z R^{-1}
        const int r = rdef;
        const size_t nr = (size_t)n * r;
        double *dw = (double *)ws_get(ctx, WS_DEFL, sizeof(double) * (4 * nr + 3 * np + (size_t)(itmax + 2) * pp +
                                                                      2 * pp + 2 * (size_t)r * r), &s);
        if (!dw) return s;
        double *Zc = dw, *Cc = dw + nr, *Qc = dw + 2 * nr, *Tc = dw + 3 * nr;
        dfl.r = r;
        dfl.Qp = dw + 4 * nr;
        dfl.Zp = dfl.Qp + np;
        dfl.Xdef = dfl.Zp + np;
        dfl.E = dfl.Xdef + np;
        dfl.E2 = dfl.E + (size_t)(itmax + 2) * pp;
        dfl.F = dfl.E2 + pp;
        double *Rr = dfl.F + pp, *Rinv = Rr + (size_t)r * r;
        BPF_TRY(colmajor_to_rowmajor(ctx, n, r, Zdef, ldz, Zc));
        BPF_TRY(spmm_rowmajor(ctx, n, A->nnz, rp, ci, av, base, r, 1.0, Zc, 0.0, Cc, nullptr));
        BPF_TRY(cholqr(ctx, n, r, Cc, Qc, Rr, Tc, st));
        std::vector<double> Rh((size_t)r * r), Ri((size_t)r * r, 0.0);
        BPF_CUDA(ctx, cudaMemcpyAsync(Rh.data(), Rr, sizeof(double) * Rh.size(), cudaMemcpyDeviceToHost, ctx->stream));
        BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        BPF_TRY(check_dev_status(ctx, "block_gmres deflation basis"));
        // Keep the leading columns whose pivots are well conditioned: a (numerically) dependent
        // column would make Z R^{-1} blow up and break A Zd = Q_C, on which the residual
        // estimate rests.  A basis with no usable column deflates nothing.
        double rmax = 0.0;
        for (int c = 0; c < r; c++) rmax = std::max(rmax, std::fabs(Rh[(size_t)c * r + c]));
        int r_ok = 0;
        while (r_ok < r && std::isfinite(Rh[(size_t)r_ok * r + r_ok]) &&
               std::fabs(Rh[(size_t)r_ok * r + r_ok]) > 1e-8 * rmax)
            r_ok++;
        for (int c = 0; c < r; c++) {   // upper-triangular inverse, column by column
            for (int i = c; i >= 0; i--) {
                double v = (i == c) ? 1.0 : 0.0;
                for (int k = i + 1; k <= c; k++) v -= Rh[(size_t)i * r + k] * Ri[(size_t)k * r + c];
                Ri[(size_t)i * r + c] = v / Rh[(size_t)i * r + i];
            }
        }
        // columns >= r_ok of Q_C and Zd are zeroed (their R^{-1} columns are dropped)
        for (int c = r_ok; c < r; c++)
            for (int i = 0; i < r; i++) Ri[(size_t)i * r + c] = 0.0;
        BPF_CUDA(ctx, cudaMemcpyAsync(Rinv, Ri.data(), sizeof(double) * Ri.size(), cudaMemcpyHostToDevice, ctx->stream));
        BPF_TRY(tsmm(ctx, n, r, 1, Zc, 0, Rinv, 0, 1.0, nullptr, 0.0, Cc, nullptr));
        const int blocks = std::max(1, std::min(ceil_div((long long)np, 256), ctx->num_sms * 8));
        // Q_C's columns from the Cholesky-QR; the dropped ones become zero columns
        pad_cols_kernel<<<blocks, 256, 0, ctx->stream>>>(n, r, p, Qc, dfl.Qp);
        BPF_LAUNCHED(ctx);
        if (r_ok < r) {
            zero_cols_kernel<<<blocks, 256, 0, ctx->stream>>>(n, r_ok, r, p, dfl.Qp);
            BPF_LAUNCHED(ctx);
        }
        pad_cols_kernel<<<blocks, 256, 0, ctx->stream>>>(n, r, p, Cc, dfl.Zp);
        BPF_LAUNCHED(ctx);
        if (r_ok == 0) dfl.r = 0;
        // keep the Cholesky-QR's retained R (its last pass) consistent: the solve only needs
        // Q_C and Zd, which satisfy A Zd = Q_C up to rounding
    }
    gmres_init_kernel<<<1, 1, 0, ctx->stream>>>(st, opts->atol, opts->rtol, hist, timemax - (now_s() - t0));
    BPF_LAUNCHED(ctx);
    BPF_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(SolveState), cudaMemcpyDeviceToHost, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));

    if (opts->verbose > 0) {
        printf("BLOCK-GMRES: system of size %d with %d right-hand sides\n", n, p);
        printf("%5s  %5s  %7s  %5s\n", "pass", "k", "‖Rₖ‖", "timer");
        printf("%5d  %5d  %7.1e  %.2fs\n", 0, 0, hs.rnorm, now_s() - t0);
    }
    int npass = 0, iter = 0, inner_itmax = itmax;
    bool solved = hs.solved != 0, tired = iter >= itmax, overtimed = false;
    int printed = 1;
    const int chunk = restart ? memory : 16;
    std::vector<double> hbuf;

    while (!(solved || tired || overtimed)) {
        pass_begin_kernel<<<1, 1, 0, ctx->stream>>>(st, inner_itmax);
        BPF_LAUNCHED(ctx);
        if (restart) {
            BPF_CUDA(ctx, cudaMemsetAsync(dX, 0, sizeof(double) * np, ctx->stream));
            if (npass >= 1) {                                               // :267-271
                BPF_TRY(spmm_rowmajor(ctx, n, A->nnz, rp, ci, av, base, p, 1.0, Xi, 0.0, W, Bi));
                if (M) BPF_TRY(prec_apply_rowmajor(ctx, M, p, W, Qm));
            }
        }
        if (dfl.r > 0) {   // R0 -= Q_C (Q_C^T R0), Xdef = Zd (Q_C^T R0)
            BPF_TRY(gram(ctx, n, p, 1, dfl.Qp, 0, R0, dfl.E2, 1.0, false, st));
            BPF_TRY(tsmm(ctx, n, p, 1, dfl.Qp, 0, dfl.E2, 0, -1.0, R0, 1.0, R0, st));
            BPF_TRY(tsmm(ctx, n, p, 1, dfl.Zp, 0, dfl.E2, 0, 1.0, nullptr, 0.0, dfl.Xdef, st));
        }
        BPF_TRY(cholqr(ctx, n, p, R0, g.V, g.Z, Tq, st));                    // :275-276
        npass++;
        const int kmax = restart ? std::min(memory, inner_itmax) : inner_itmax;
        int k = 0;
        bool active = true;
        while (active && k < kmax) {
            const int kend = std::min(kmax, k + chunk);
            if (kend > g.cap) {
                int newcap = std::min(std::max(kend, 2 * g.cap), std::max(kmax, 1));
                BPF_TRY(gmres_capacity(ctx, n, p, newcap, g.cap, g, flexible));
            }
            // Size the Gram workspaces for the largest k of this chunk up front, so no
            // allocation (and no implicit synchronisation) happens between launches.
            double *Psi2buf = (double *)ws_get(ctx, WS_I32, sizeof(double) * pp * kend, &s);
            if (!Psi2buf) return s;
            if (!ws_get(ctx, WS_PARTIAL, sizeof(double) * pp * ((size_t)ctx->num_sms * 4 + kend + 1), &s))
                return s;
            for (int kk = k + 1; kk <= kend; kk++) {
                const int jj = kk - 1;
                double *Vk = g.V + (size_t)jj * np;
                double *Vn = g.V + (size_t)kk * np;
                const double *Pk = Vk;
                if (N) {                                                     // :297-298
                    double *dst = flexible ? g.Zb + (size_t)jj * np : Pm;
                    BPF_TRY(prec_apply_rowmajor(ctx, N, p, Vk, dst, &st->active));
                    Pk = dst;
                }
                BPF_TRY(spmm_rowmajor(ctx, n, A->nnz, rp, ci, av, base, p, 1.0, Pk, 0.0, W, nullptr, &st->active));
                double *Qk = W;
                if (M) {                                                     // :300
                    BPF_TRY(prec_apply_rowmajor(ctx, M, p, W, Qm, &st->active));
                    Qk = Qm;
                }
                double *Psi = g.Rblk + rblk_pos(0, jj) * pp;                     // :301-313
                double *Ek = dfl.r > 0 ? dfl.E + (size_t)jj * pp : nullptr;
                if (Ek) {   // against Q_C first (GCRO): E_k = Q_C^T W, W -= Q_C E_k
                    BPF_TRY(gram(ctx, n, p, 1, dfl.Qp, 0, Qk, Ek, 1.0, false, st));
                    BPF_TRY(tsmm(ctx, n, p, 1, dfl.Qp, 0, Ek, 0, -1.0, Qk, 1.0, Qk, st));
                }
                BPF_TRY(gram(ctx, n, p, kk, g.V, np, Qk, Psi, 1.0, false, st));
                BPF_TRY(tsmm(ctx, n, p, kk, g.V, np, Psi, pp, -1.0, Qk, 1.0, Qk, st));
                if (Ek) {
                    BPF_TRY(gram(ctx, n, p, 1, dfl.Qp, 0, Qk, Ek, 1.0, true, st, nullptr, dfl.E2));
                    BPF_TRY(tsmm(ctx, n, p, 1, dfl.Qp, 0, dfl.E2, 0, -1.0, Qk, 1.0, Qk, st));
                }
                BPF_TRY(gram(ctx, n, p, kk, g.V, np, Qk, Psi, 1.0, true, st, nullptr, Psi2buf));
                BPF_TRY(tsmm(ctx, n, p, kk, g.V, np, Psi2buf, pp, -1.0, Qk, 1.0, Qk, st));
                double *Cm = Cpar[kk & 1];
                // Cpar[kk & 1] was last read by the Hessenberg update of iteration kk - 2
                if (overlap && kk >= 3)
                    BPF_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_b[kk & 1], 0));
                BPF_TRY(cholqr(ctx, n, p, Qk, Vn, Cm, Tq, st, nullptr, &st->qr_shift,
                               &st->qr_reorth, kk));                         // :316
                // Ill-conditioned block (Cholesky lost > 8 digits): its Q may carry amplified
                // components along V.  Re-orthogonalize once and fold the correction into the
                // Hessenberg column: W = V Psi + Q1 R1, Q1 = V Phi + Q2 C2
                //   => Psi += Phi R1, C = C2 R1.  Gated on the device flag.
                {
                    const int *rg = &st->qr_reorth;
                    BPF_TRY(gram(ctx, n, p, kk, g.V, np, Vn, Psi2buf, 1.0, false, st, rg));
                    BPF_TRY(tsmm(ctx, n, p, kk, g.V, np, Psi2buf, pp, -1.0, Vn, 1.0, Qk, st, nullptr, rg));
                    BPF_TRY(cholqr(ctx, n, p, Qk, Vn, C2, Tq, st, rg, &st->qr_shift2, nullptr, kk));
                    BPF_TRY(reorth_fold(ctx, p, kk, Psi, Psi2buf, Cm, C2, Cm, fold_scr, st, rg));
                }
                if (overlap) {
                    BPF_CUDA(ctx, cudaEventRecord(ctx->ev_a[kk & 1], ctx->stream));
                    BPF_CUDA(ctx, cudaStreamWaitEvent(ctx->hstream, ctx->ev_a[kk & 1], 0));
                    StreamSwap sw(ctx, ctx->hstream);
                    BPF_TRY(launch_hess(ctx, p, kk, g.Rblk, g.HY, tau_cur, g.Z, Cm, st, hist, scr));
                    BPF_CUDA(ctx, cudaEventRecord(ctx->ev_b[kk & 1], ctx->hstream));
                    last_hess = kk;
                } else {
                    BPF_TRY(launch_hess(ctx, p, kk, g.Rblk, g.HY, tau_cur, g.Z, Cm, st, hist, scr));
                }
            }
            k = kend;
            BPF_TRY(join());
            BPF_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(SolveState), cudaMemcpyDeviceToHost, ctx->stream));
            BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            // a Cholesky-QR breakdown in an iteration that counted is an error (one in an
            // iteration past the stopping point is not)
            if (hs.qr_fail_iter <= hs.inner_iter)
                return set_error(ctx, BPF_ERR_NUMERIC, "block_gmres: Cholesky-QR breakdown");
            active = hs.active != 0;
            if (opts->verbose > 0 && hs.nres > printed) {
                int upto = std::min(hs.nres, hist_cap);
                hbuf.resize(upto);
                BPF_CUDA(ctx, cudaMemcpy(hbuf.data(), hist, sizeof(double) * upto, cudaMemcpyDeviceToHost));
                for (int q = printed; q < upto; q++) {
                    const int it = q;  // cumulative iteration index of residual q
                    if (it % opts->verbose == 0)
                        printf("%5d  %5d  %7.1e  %.2fs\n", npass, it, hbuf[q], now_s() - t0);
                }
                printed = upto;
            }
            if (now_s() - t0 > timemax) break;
        }
        const int inner_iter = hs.inner_iter;
        // :366-385
        double *Yb = (double *)ws_get(ctx, WS_Y, sizeof(double) * pp * std::max(inner_iter, 1), &s);
        if (!Yb) return s;
        BPF_TRY(launch_backsub(ctx, p, inner_iter, g.Rblk, g.HY, g.Z, Yb));
        if (flexible) {                                                     // X += sum (N \ V_i) Y_i
            BPF_TRY(tsmm(ctx, n, p, inner_iter, g.Zb, np, Yb, pp, 1.0, Xr, 1.0, Xr, nullptr));
        } else {
            BPF_TRY(tsmm(ctx, n, p, inner_iter, g.V, np, Yb, pp, 1.0, Xr, 1.0, Xr, nullptr));
        }
        if (N && !flexible) {
            BPF_CUDA(ctx, cudaMemcpyAsync(Pm, Xr, sizeof(double) * np, cudaMemcpyDeviceToDevice, ctx->stream));
            BPF_TRY(prec_apply_rowmajor(ctx, N, p, Pm, Xr));
        }
        if (dfl.r > 0 && inner_iter > 0) {   // x = x0' + N^{-1} V y - Zd (E y)
            BPF_TRY(tsmm(ctx, p, p, inner_iter, dfl.E, pp, Yb, pp, 1.0, nullptr, 0.0, dfl.F, nullptr));
            BPF_TRY(tsmm(ctx, n, p, 1, dfl.Zp, 0, dfl.F, 0, -1.0, dfl.Xdef, 1.0, dfl.Xdef, nullptr));
        }
        if (dfl.r > 0) BPF_TRY(axpby(ctx, np, 1.0, dfl.Xdef, 1.0, Xr, nullptr));
        if (restart) BPF_TRY(axpby(ctx, np, 1.0, dX, 1.0, Xi, nullptr));
        inner_itmax -= inner_iter;                                          // :388-392
        iter += inner_iter;
        tired = iter >= itmax;
        solved = hs.solved != 0;
        overtimed = hs.overtimed != 0 || (now_s() - t0 > timemax);
        if (inner_iter == 0) break;  // nothing progressed (time limit hit before the first iteration)
    }
    if (warm && !restart) BPF_TRY(axpby(ctx, np, 1.0, dX, 1.0, Xi, nullptr));   // :402
    BPF_TRY(rowmajor_to_colmajor(ctx, n, p, Xi, X, ldx));
    BPF_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(SolveState), cudaMemcpyDeviceToHost, ctx->stream));
    BPF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    BPF_TRY(check_dev_status(ctx, "block_gmres"));
    int status = BPF_SOLVE_UNKNOWN;                                          // :397-399
    if (tired) status = BPF_SOLVE_ITMAX;
    if (solved) status = BPF_SOLVE_SOLVED;
    if (overtimed) status = BPF_SOLVE_TIMEMAX;
    stats->niter = iter;
    stats->solved = solved;
    stats->status = status;
    stats->npass = npass;
    stats->n_residuals = opts->history ? std::min(hs.nres, hist_cap) : 0;
    if (opts->history && stats->residuals && stats->residuals_capacity > 0) {
        int cnt = std::min(stats->n_residuals, stats->residuals_capacity);
        BPF_CUDA(ctx, cudaMemcpy(stats->residuals, hist, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
    }
    if (opts->verbose > 0) printf("\n");
    stats->timer = now_s() - t0;
    return BPF_SUCCESS;
}

// Blocks wider than the 128 columns one solve takes are solved in column slices of at most 128
// (nearly equal widths), each by block-GMRES with atol scaled by sqrt(p_s / p): by Minkowski's
// inequality the slices' residuals then meet ||R||_F <= atol + rtol ||B||_F for the whole block,
// the reference's test (src/block_gmres.jl:223-231).  itmax defaults to 2 div(n, p) of the whole
// block.  Stats: niter and npass are the slices' largest, solved = every slice solved, the
// residual history at iteration k the root-sum-square of the slices' (a finished slice keeps its
// last value), timer the sum.
static bpf_status block_gmres_sliced(bpf_ctx *ctx, const bpf_csr_desc *A, int p, const double *B, int ldb,
                                     double *X, int ldx, const double *X0, int ldx0, const bpf_prec *M,
                                     const bpf_prec *N, const bpf_gmres_opts *opts, bpf_stats *stats) {
    const int ns = (p + 127) / 128;
    const int n = A->n;
    bpf_gmres_opts o = *opts;
    if (o.itmax == 0) o.itmax = std::max(1, 2 * (n / p));
    const int cap = o.itmax + 2;
    std::vector<std::vector<double>> hist(ns, std::vector<double>(cap, 0.0));
    std::vector<int> nres(ns, 0);
    int niter = 0, npass = 0, solved = 1, status = BPF_SOLVE_SOLVED;
    double timer = 0.0;
    int c0 = 0;
    for (int k = 0; k < ns; k++) {
        const int q = p / ns + (k < p % ns ? 1 : 0);
        bpf_gmres_opts os = o;
        os.atol = o.atol * std::sqrt((double)q / (double)p);
        if (o.timemax > 0.0 && o.timemax < 1e300) os.timemax = std::max(1e-9, o.timemax - timer);
        bpf_stats st{};
        st.residuals_capacity = cap;
        st.residuals = hist[k].data();
        bpf_status r = block_gmres_impl(ctx, A, q, B + (size_t)c0 * ldb, ldb, X + (size_t)c0 * ldx, ldx,
                                        X0 ? X0 + (size_t)c0 * ldx0 : nullptr, ldx0, M, N, &os, &st, nullptr, 0, 0);
        if (r != BPF_SUCCESS) return r;
        niter = std::max(niter, st.niter);
        npass = std::max(npass, st.npass);
        timer += st.timer;
        nres[k] = std::min(st.n_residuals, cap);
        if (!st.solved) {
            solved = 0;
            if (st.status == BPF_SOLVE_TIMEMAX || status == BPF_SOLVE_TIMEMAX) status = BPF_SOLVE_TIMEMAX;
            else status = st.status;
        }
        c0 += q;
    }
    if (stats) {
        stats->niter = niter;
        stats->solved = solved;
        stats->status = status;
        stats->timer = timer;
        stats->npass = npass;
        int nr = 0;
        for (int k = 0; k < ns; k++) nr = std::max(nr, nres[k]);
        stats->n_residuals = nr;
        if (stats->residuals && stats->residuals_capacity > 0) {
            for (int i = 0; i < std::min(nr, stats->residuals_capacity); i++) {
                double s2 = 0.0;
                for (int k = 0; k < ns; k++) {
                    if (nres[k] == 0) continue;
                    const double v = hist[k][std::min(i, nres[k] - 1)];
                    s2 += v * v;
                }
                stats->residuals[i] = std::sqrt(s2);
            }
        }
    }
    return BPF_SUCCESS;
}

extern "C" bpf_status bpf_block_gmres(bpf_ctx *ctx, const bpf_csr_desc *A, int p, const double *B,
                                      int ldb, double *X, int ldx, const double *X0, int ldx0,
                                      const bpf_prec *M, const bpf_prec *N, const bpf_gmres_opts *opts,
                                      bpf_stats *stats) {
    if (ctx && A && opts && B && X && p > 128 && p <= A->n)
        return block_gmres_sliced(ctx, A, p, B, ldb, X, ldx, X0, ldx0, M, N, opts, stats);
    return block_gmres_impl(ctx, A, p, B, ldb, X, ldx, X0, ldx0, M, N, opts, stats, nullptr, 0, 0);
}

extern "C" bpf_status bpf_block_gmres_deflated(bpf_ctx *ctx, const bpf_csr_desc *A, int p,
                                               const double *B, int ldb, double *X, int ldx,
                                               const double *X0, int ldx0, const bpf_prec *M,
                                               const bpf_prec *N, const bpf_gmres_opts *opts,
                                               const double *Z, int ldz, int rank, bpf_stats *stats) {
    if (rank < 0) return set_error(ctx, BPF_ERR_INVALID_VALUE, "block_gmres: negative deflation rank");
    return block_gmres_impl(ctx, A, p, B, ldb, X, ldx, X0, ldx0, M, N, opts, stats, Z, ldz, rank);
}
