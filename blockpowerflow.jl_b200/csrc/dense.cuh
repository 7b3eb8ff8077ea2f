// Dense block kernels on row-major n x p blocks and p x p small matrices (row-major).
#pragma once

#include "bpf_internal.cuh"

namespace bpf {

// Device state shared by the kernels of one Krylov solve (GMRES and BiCGSTAB).
struct SolveState {
    int active;        // 1 while the current pass continues; kernels no-op when 0
    int inner_iter;    // iterations done in the current pass
    int iter;          // cumulative iterations
    int solved;
    int inner_tired;
    int overtimed;
    int itmax;
    int inner_itmax;
    int mem;
    int restart;
    int nres;          // residual norms written to the history buffer
    int hist_cap;
    int qr_shift;      // a Cholesky-QR pass needed the shift (third pass runs)
    int qr_fail;
    int qr_reorth;     // the new basis block was ill-conditioned: re-orthogonalize it
    int qr_shift2;     // shift flag of the re-orthogonalization's Cholesky-QR
    int qr_fail_iter;  // smallest tagged iteration whose Cholesky-QR broke down (INT_MAX: none)
    int pad1;
    double eps;
    double rnorm;
    double atol, rtol;
    double omega;      // BiCGSTAB
    unsigned long long deadline_ns;  // %globaltimer deadline (0 = none)
    double pad2[4];
};

// Out_j (p x p) = alpha * A_j^T B, j = 0..nb-1, A_j = A + j*strideA (row-major n x p).
// Reduced over n in two deterministic stages through the WS_PARTIAL workspace.
// accumulate: Out_j += result instead of =.  st (nullable): skip when !st->active.
// Out2 (nullable): also receives the new result itself (before accumulation).
bpf_status gram(bpf_ctx *ctx, int n, int p, int nb, const double *A, size_t strideA,
                const double *B, double *Out, double alpha, bool accumulate,
                const SolveState *st, const int *qr_gate = nullptr, double *Out2 = nullptr,
                const int *gate2 = nullptr);

// Out = beta*Cin + alpha * sum_{j<nb} A_j S_j  (A_j row-major n x p, S_j p x p row-major).
// Cin may be nullptr (treated as 0) or equal Out.  Out must not alias any A_j.
// nb_dev (nullable): read the number of blocks from device memory (<= nb).
bpf_status tsmm(bpf_ctx *ctx, int n, int p, int nb, const double *A, size_t strideA,
                const double *S, size_t strideS, double alpha, const double *Cin, double beta,
                double *Out, const SolveState *st, const int *nb_dev = nullptr,
                const int *qr_gate = nullptr, const int *gate2 = nullptr);

// Cholesky-QR of W (n x p) into Q (n x p, distinct buffer), R (p x p upper, row-major).
// Two passes, plus a shifted first pass and a third pass when the Gram matrix is not
// numerically positive definite (rank-deficient / ill-conditioned blocks).
//   gate (nullable): every kernel is skipped when *gate == 0.
//   shift_flag: set by the first pass when it needed the shift (default st->qr_shift).
//   reorth_flag (nullable): set when the first Cholesky lost more than 8 digits on some
//   column (the block was ill-conditioned; its Q should be re-orthogonalized).
//   iter_tag >= 0: a breakdown records min(st->qr_fail_iter, iter_tag) instead of raising the
//   context's device error (block-GMRES decides on the host whether that iteration counted).
bpf_status cholqr(bpf_ctx *ctx, int n, int p, const double *W, double *Q, double *R,
                  double *tmp_block, SolveState *st, const int *gate = nullptr,
                  int *shift_flag = nullptr, int *reorth_flag = nullptr, int iter_tag = -1);

// Psi_i += Phi_i R1 (i < nb), C <- C2 R1: folds a re-orthogonalization of the basis block
// into the Hessenberg column.  Gated by *gate.
bpf_status reorth_fold(bpf_ctx *ctx, int p, int nb, double *Psi, const double *Phi,
                       const double *R1, const double *C2, double *C, double *scratch,
                       const SolveState *st, const int *gate);

// Elementwise helpers on n*p doubles.
bpf_status axpby(bpf_ctx *ctx, size_t len, double a, const double *x, double b, double *y,
                 const SolveState *st);  // y = a*x + b*y
bpf_status frob_norm(bpf_ctx *ctx, size_t len, const double *x, double *out);  // device scalar

}  // namespace bpf
