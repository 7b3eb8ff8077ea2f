/*
 * bpf_oracle.c -- CPU restatement of the reference's multi-RHS sparse solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke entry and the
 * bench's CPU-baseline leg call it through ctypes.  The shipped library never links it,
 * and nothing on the product path falls back to it.
 *
 * Every routine restates one piece of exanauts/BlockPowerFlow.jl (Julia, FP64):
 *   - orc_spmm             mul!(Y, A, X, a, b) on CSR                (src/block_gmres.jl:299)
 *   - orc_ilu0             csrilu02 semantics: ILU(0) on A's pattern  (src/preconditioners_nvidia.jl:42-47)
 *   - orc_ic0              csric02 semantics: IC(0) on A's lower part (src/preconditioners_nvidia.jl:6-11)
 *   - orc_prec_apply       ldiv!(y, P, x) for ILU0 / IC0              (src/preconditioners_nvidia.jl:13-35,55-58)
 *   - orc_householder      householder!(Q, R, tau; compact)          (src/block_utils.jl:46-53)
 *   - orc_block_gmres      block_gmres!                              (src/block_gmres.jl:170-411)
 *   - orc_block_bicgstab   CPU block_bicgstab!                       (src/block_bicgstab.jl:70-178)
 *   - orc_lu_*             host LU + refactor-on-fixed-pivots + solve (src/cusolverRF.jl:56-331),
 *                          dense, for the small cases the oracle has to finish in seconds.
 *
 * Pinning (tests/test_oracle.py, fixtures from the reference's data by tests/golden/make_golden.py):
 * the RF routines against the reference's four cusolverRF known-answer tests (test/cusolverRF.jl),
 * ILU(0) / IC(0) against exact factorizations on patterns without fill, the Householder QR
 * against LAPACK's conventions.  The block solvers are pinned to the reference tests' settings
 * and to the direct solve only: their iteration counts and histories are parity unpinned, since
 * the reference's block-solver tests only print and the reference cannot run here (no Julia).
 *
 * Dense blocks are column-major with an explicit leading dimension, like Julia matrices.
 * CSR arrays are 0-based int32.  Parallelism (OpenMP) only splits independent loops
 * (rows of a SpMM, RHS columns of a triangular solve, columns of a reflector update) so the
 * arithmetic per output element is the same sequential sum at any thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR_DIM 2
#define ORC_ERR_ALLOC 4
#define ORC_ERR_SINGULAR 5

/* ------------------------------------------------------------------------------------- */
/* threads                                                                                 */
/* ------------------------------------------------------------------------------------- */
static int g_threads = 1;
void orc_set_threads(int t) { g_threads = t < 1 ? 1 : t; }
int orc_get_threads(void) { return g_threads; }

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* ------------------------------------------------------------------------------------- */
/* sparse kernels                                                                          */
/* ------------------------------------------------------------------------------------- */

/* Y = alpha*A*X + beta*Y ; A n x n CSR, X/Y n x p column-major.  (src/block_gmres.jl:299) */
void orc_spmm(int n, const int *rp, const int *ci, const double *v, int p, double alpha,
              const double *X, int ldx, double beta, double *Y, int ldy) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int i = 0; i < n; i++) {
        for (int c = 0; c < p; c++) {
            double s = 0.0;
            for (int k = rp[i]; k < rp[i + 1]; k++) s += v[k] * X[(size_t)c * ldx + ci[k]];
            double y = alpha * s;
            if (beta != 0.0) y += beta * Y[(size_t)c * ldy + i];
            Y[(size_t)c * ldy + i] = y;
        }
    }
}

static int find_diag(int n, const int *rp, const int *ci, int *diag) {
    for (int i = 0; i < n; i++) {
        diag[i] = -1;
        for (int k = rp[i]; k < rp[i + 1]; k++)
            if (ci[k] == i) { diag[i] = k; break; }
        if (diag[i] < 0) return -(i + 1);
    }
    return 0;
}

/* ILU(0) in place on A's pattern, IKJ order, unit-lower L and upper U sharing the CSR
 * (csrilu02 as called by ilu0(), src/preconditioners_nvidia.jl:42-47).  Column indices of
 * each row must be sorted.  Returns 0, or -(i+1) for a structurally missing or zero pivot. */
int orc_ilu0(int n, const int *rp, const int *ci, double *v) {
    int *diag = (int *)malloc(sizeof(int) * n);
    int *pos = (int *)malloc(sizeof(int) * n);
    if (!diag || !pos) { free(diag); free(pos); return ORC_ERR_ALLOC; }
    int st = find_diag(n, rp, ci, diag);
    if (st) { free(diag); free(pos); return st; }
    for (int j = 0; j < n; j++) pos[j] = -1;
    for (int i = 0; i < n && st == 0; i++) {
        for (int k = rp[i]; k < rp[i + 1]; k++) pos[ci[k]] = k;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            int kc = ci[k];
            if (kc >= i) break;
            double piv = v[diag[kc]];
            if (piv == 0.0) { st = -(kc + 1); break; }
            double lik = v[k] / piv;
            v[k] = lik;
            for (int j = diag[kc] + 1; j < rp[kc + 1]; j++) {
                int q = pos[ci[j]];
                if (q >= 0) v[q] -= lik * v[j];
            }
        }
        for (int k = rp[i]; k < rp[i + 1]; k++) pos[ci[k]] = -1;
        if (st == 0 && v[diag[i]] == 0.0) st = -(i + 1);
    }
    free(diag);
    free(pos);
    return st;
}

/* IC(0) in place on the lower triangle of A's pattern (upper part left untouched),
 * csric02 as called by ic0() (src/preconditioners_nvidia.jl:6-11).  Up-looking:
 * l_ik = (a_ik - sum_{j<k} l_ij l_kj) / l_kk,  l_ii = sqrt(a_ii - sum_{j<i} l_ij^2).
 * Returns -(i+1) when a pivot is not positive. */
int orc_ic0(int n, const int *rp, const int *ci, double *v) {
    int *diag = (int *)malloc(sizeof(int) * n);
    int *pos = (int *)malloc(sizeof(int) * n);
    if (!diag || !pos) { free(diag); free(pos); return ORC_ERR_ALLOC; }
    int st = find_diag(n, rp, ci, diag);
    if (st) { free(diag); free(pos); return st; }
    for (int j = 0; j < n; j++) pos[j] = -1;
    for (int i = 0; i < n && st == 0; i++) {
        for (int k = rp[i]; k < rp[i + 1]; k++) pos[ci[k]] = k;
        for (int k = rp[i]; k < diag[i]; k++) {
            int kc = ci[k];
            double s = v[k];
            /* sum over j < kc present in both row i and row kc */
            for (int j = rp[kc]; j < diag[kc]; j++) {
                int q = pos[ci[j]];
                if (q >= 0) s -= v[q] * v[j];
            }
            v[k] = s / v[diag[kc]];
        }
        double d = v[diag[i]];
        for (int k = rp[i]; k < diag[i]; k++) d -= v[k] * v[k];
        if (!(d > 0.0)) st = -(i + 1);
        else v[diag[i]] = sqrt(d);
        for (int k = rp[i]; k < rp[i + 1]; k++) pos[ci[k]] = -1;
    }
    free(diag);
    free(pos);
    return st;
}

/* Triangular solves on a CSR factor, p columns (column-major), X may alias Y.
 * kind 0: unit lower L (strict lower part)        -- ILU0 forward  (UnitLowerTriangular)
 * kind 1: upper U incl. diagonal                   -- ILU0 backward (UpperTriangular)
 * kind 2: lower L incl. diagonal                   -- IC0 forward   (LowerTriangular)
 * kind 3: transpose of lower L incl. diagonal      -- IC0 backward  (LowerTriangular')  */
void orc_trsm(int kind, int n, const int *rp, const int *ci, const double *v, int p,
              const double *X, int ldx, double *Y, int ldy) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int c = 0; c < p; c++) {
        const double *x = X + (size_t)c * ldx;
        double *y = Y + (size_t)c * ldy;
        if (x != y) memcpy(y, x, sizeof(double) * n);
        if (kind == 0) {
            for (int i = 0; i < n; i++) {
                double s = y[i];
                for (int k = rp[i]; k < rp[i + 1] && ci[k] < i; k++) s -= v[k] * y[ci[k]];
                y[i] = s;
            }
        } else if (kind == 1) {
            for (int i = n - 1; i >= 0; i--) {
                double s = y[i], d = 0.0;
                for (int k = rp[i]; k < rp[i + 1]; k++) {
                    if (ci[k] > i) s -= v[k] * y[ci[k]];
                    else if (ci[k] == i) d = v[k];
                }
                y[i] = s / d;
            }
        } else if (kind == 2) {
            for (int i = 0; i < n; i++) {
                double s = y[i], d = 0.0;
                for (int k = rp[i]; k < rp[i + 1]; k++) {
                    if (ci[k] < i) s -= v[k] * y[ci[k]];
                    else if (ci[k] == i) d = v[k];
                }
                y[i] = s / d;
            }
        } else {
            for (int i = n - 1; i >= 0; i--) {
                double d = 0.0;
                for (int k = rp[i]; k < rp[i + 1]; k++)
                    if (ci[k] == i) d = v[k];
                double yi = y[i] / d;
                y[i] = yi;
                for (int k = rp[i]; k < rp[i + 1] && ci[k] < i; k++) y[ci[k]] -= v[k] * yi;
            }
        }
    }
}

/* Preconditioner operator: kind 0 none (identity), 1 ILU0 factors, 2 IC0 factors. */
typedef struct {
    int kind;
    int n;
    const int *rp, *ci;
    const double *v;
} orc_prec;

/* y = P \ x  (ldiv! of src/preconditioners_nvidia.jl:13-35 and :55-58; scratch z inside). */
static void prec_apply(const orc_prec *P, int p, const double *X, int ldx, double *Y, int ldy) {
    int n = P->n;
    if (P->kind == 0) {
        for (int c = 0; c < p; c++)
            if (X + (size_t)c * ldx != Y + (size_t)c * ldy)
                memcpy(Y + (size_t)c * ldy, X + (size_t)c * ldx, sizeof(double) * n);
        return;
    }
    double *z = (double *)malloc(sizeof(double) * (size_t)n * p);
    if (P->kind == 1) {
        orc_trsm(0, n, P->rp, P->ci, P->v, p, X, ldx, z, n);
        orc_trsm(1, n, P->rp, P->ci, P->v, p, z, n, Y, ldy);
    } else {
        orc_trsm(2, n, P->rp, P->ci, P->v, p, X, ldx, z, n);
        orc_trsm(3, n, P->rp, P->ci, P->v, p, z, n, Y, ldy);
    }
    free(z);
}

void orc_prec_apply(int kind, int n, const int *rp, const int *ci, const double *v, int p,
                    const double *X, int ldx, double *Y, int ldy) {
    orc_prec P = {kind, n, rp, ci, v};
    prec_apply(&P, p, X, ldx, Y, ldy);
}

/* ------------------------------------------------------------------------------------- */
/* dense helpers (column-major)                                                            */
/* ------------------------------------------------------------------------------------- */
#define AT(A, ld, i, j) (A)[(size_t)(j) * (ld) + (i)]

/* Cache-blocked products, switched on only to time the oracle as the CPU baseline (the checker
 * keeps the plain loops below, so its rounding does not change): the same sums in another order. */
static int g_fast_dense = 0;
void orc_set_fast_dense(int on) { g_fast_dense = on != 0; }

/* C = alpha A^T B + beta C, A k x m, B k x ncol: the k range split over the threads, each summing
 * a private m x ncol block in 4 x 4 register tiles (16 independent sums per row of A and B). */
static void gemm_tn_blocked(int m, int ncol, int k, double alpha, const double *A, int lda,
                            const double *B, int ldb, double beta, double *C, int ldc) {
    const int T = g_threads;
    double *part = (double *)calloc((size_t)T * m * ncol, sizeof(double));
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const int l0 = (int)((long long)k * t / nt), l1 = (int)((long long)k * (t + 1) / nt);
        double *P = part + (size_t)t * m * ncol;
        for (int j0 = 0; j0 < ncol; j0 += 4) {
            const int jb = ncol - j0 < 4 ? ncol - j0 : 4;
            for (int i0 = 0; i0 < m; i0 += 4) {
                const int ib = m - i0 < 4 ? m - i0 : 4;
                double acc[4][4] = {{0}};
                if (ib == 4 && jb == 4) {
                    const double *a0 = A + (size_t)i0 * lda, *a1 = a0 + lda, *a2 = a1 + lda, *a3 = a2 + lda;
                    const double *b0 = B + (size_t)j0 * ldb, *b1 = b0 + ldb, *b2 = b1 + ldb, *b3 = b2 + ldb;
                    for (int l = l0; l < l1; l++) {
                        const double x0 = a0[l], x1 = a1[l], x2 = a2[l], x3 = a3[l];
                        const double y0 = b0[l], y1 = b1[l], y2 = b2[l], y3 = b3[l];
                        acc[0][0] += x0 * y0; acc[0][1] += x0 * y1; acc[0][2] += x0 * y2; acc[0][3] += x0 * y3;
                        acc[1][0] += x1 * y0; acc[1][1] += x1 * y1; acc[1][2] += x1 * y2; acc[1][3] += x1 * y3;
                        acc[2][0] += x2 * y0; acc[2][1] += x2 * y1; acc[2][2] += x2 * y2; acc[2][3] += x2 * y3;
                        acc[3][0] += x3 * y0; acc[3][1] += x3 * y1; acc[3][2] += x3 * y2; acc[3][3] += x3 * y3;
                    }
                } else {
                    for (int ii = 0; ii < ib; ii++)
                        for (int jj = 0; jj < jb; jj++) {
                            const double *a = A + (size_t)(i0 + ii) * lda, *b = B + (size_t)(j0 + jj) * ldb;
                            double s2 = 0.0;
                            for (int l = l0; l < l1; l++) s2 += a[l] * b[l];
                            acc[ii][jj] = s2;
                        }
                }
                for (int ii = 0; ii < ib; ii++)
                    for (int jj = 0; jj < jb; jj++) P[(size_t)(j0 + jj) * m + i0 + ii] = acc[ii][jj];
            }
        }
    }
    for (int j = 0; j < ncol; j++)
        for (int i = 0; i < m; i++) {
            double s2 = 0.0;
            for (int t = 0; t < T; t++) s2 += part[(size_t)t * m * ncol + (size_t)j * m + i];
            AT(C, ldc, i, j) = alpha * s2 + (beta == 0.0 ? 0.0 : beta * AT(C, ldc, i, j));
        }
    free(part);
}

/* C = alpha A B + beta C, A m x k, B k x ncol: blocks of 256 rows over the threads, each column
 * of C updated by contiguous column streams of A (axpy form). */
static void gemm_nn_blocked(int m, int ncol, int k, double alpha, const double *A, int lda,
                            const double *B, int ldb, double beta, double *C, int ldc) {
    const int nblk = (m + 255) / 256;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int b = 0; b < nblk; b++) {
        const int i0 = b * 256, i1 = i0 + 256 < m ? i0 + 256 : m;
        for (int j = 0; j < ncol; j++) {
            double *c = C + (size_t)j * ldc;
            if (beta == 0.0)
                for (int i = i0; i < i1; i++) c[i] = 0.0;
            else if (beta != 1.0)
                for (int i = i0; i < i1; i++) c[i] *= beta;
            for (int l = 0; l < k; l++) {
                const double w = alpha * AT(B, ldb, l, j);
                const double *a = A + (size_t)l * lda;
                for (int i = i0; i < i1; i++) c[i] += w * a[i];
            }
        }
    }
}

/* C = alpha * op(A) * B + beta * C ; op = A or A^T.  A is (ta? k x m : m x k). */
static void gemm(int ta, int m, int ncol, int k, double alpha, const double *A, int lda,
                 const double *B, int ldb, double beta, double *C, int ldc) {
    if (g_fast_dense && (size_t)m * ncol * k > 200000) {
        if (ta) gemm_tn_blocked(m, ncol, k, alpha, A, lda, B, ldb, beta, C, ldc);
        else gemm_nn_blocked(m, ncol, k, alpha, A, lda, B, ldb, beta, C, ldc);
        return;
    }
#pragma omp parallel for num_threads(g_threads) schedule(static) if ((size_t)m * ncol * k > 200000)
    for (int j = 0; j < ncol; j++) {
        for (int i = 0; i < m; i++) {
            double s = 0.0;
            if (ta) {
                for (int l = 0; l < k; l++) s += AT(A, lda, l, i) * AT(B, ldb, l, j);
            } else {
                for (int l = 0; l < k; l++) s += AT(A, lda, i, l) * AT(B, ldb, l, j);
            }
            AT(C, ldc, i, j) = alpha * s + (beta == 0.0 ? 0.0 : beta * AT(C, ldc, i, j));
        }
    }
}

/* geqrf: Householder QR in place (LAPACK dlarfg conventions: beta = -sign(alpha)*norm,
 * tau = (beta - alpha)/beta, v(1) = 1, R diagonal may be negative). */
static void geqrf(int m, int k, double *A, int lda, double *tau) {
    for (int j = 0; j < k; j++) {
        double alpha = AT(A, lda, j, j);
        double xn = 0.0;
        for (int i = j + 1; i < m; i++) xn += AT(A, lda, i, j) * AT(A, lda, i, j);
        xn = sqrt(xn);
        if (xn == 0.0) {
            tau[j] = 0.0;
            continue;
        }
        double beta = -copysign(hypot(alpha, xn), alpha);
        tau[j] = (beta - alpha) / beta;
        double scal = 1.0 / (alpha - beta);
        for (int i = j + 1; i < m; i++) AT(A, lda, i, j) *= scal;
        AT(A, lda, j, j) = beta;
        double tj = tau[j];
#pragma omp parallel for num_threads(g_threads) schedule(static) if ((size_t)m * (k - j) > 100000)
        for (int c = j + 1; c < k; c++) {
            double w = AT(A, lda, j, c);
            for (int i = j + 1; i < m; i++) w += AT(A, lda, i, j) * AT(A, lda, i, c);
            w *= tj;
            AT(A, lda, j, c) -= w;
            for (int i = j + 1; i < m; i++) AT(A, lda, i, c) -= w * AT(A, lda, i, j);
        }
    }
}

/* Apply H_j = I - tau_j v_j v_j^T (v_j stored below the diagonal of column j of A). */
static void apply_reflector(int m, int j, const double *A, int lda, double tj, double *C,
                            int ldc, int ncol) {
    if (tj == 0.0) return;
#pragma omp parallel for num_threads(g_threads) schedule(static) if ((size_t)m * ncol > 100000)
    for (int c = 0; c < ncol; c++) {
        double w = AT(C, ldc, j, c);
        for (int i = j + 1; i < m; i++) w += AT(A, lda, i, j) * AT(C, ldc, i, c);
        w *= tj;
        AT(C, ldc, j, c) -= w;
        for (int i = j + 1; i < m; i++) AT(C, ldc, i, c) -= w * AT(A, lda, i, j);
    }
}

/* orgqr: overwrite the reflectors with the explicit m x k orthonormal Q. */
static void orgqr(int m, int k, double *A, int lda, const double *tau) {
    double *Q = (double *)calloc((size_t)m * k, sizeof(double));
    for (int j = 0; j < k; j++) AT(Q, m, j, j) = 1.0;
    for (int j = k - 1; j >= 0; j--) apply_reflector(m, j, A, lda, tau[j], Q, m, k);
    for (int j = 0; j < k; j++) memcpy(&AT(A, lda, 0, j), &AT(Q, m, 0, j), sizeof(double) * m);
    free(Q);
}

/* ormqr('L','T'): C <- Q^T C with Q = H_1 ... H_k. */
static void ormqr_lt(int m, int k, const double *A, int lda, const double *tau, double *C,
                     int ldc, int ncol) {
    for (int j = 0; j < k; j++) apply_reflector(m, j, A, lda, tau[j], C, ldc, ncol);
}

/* householder!(Q, R, tau; compact) (src/block_utils.jl:46-53). */
void orc_householder(int m, int k, double *Q, int ldq, double *R, int ldr, double *tau,
                     int compact) {
    for (int j = 0; j < k; j++)
        for (int i = 0; i < k; i++) AT(R, ldr, i, j) = 0.0;
    geqrf(m, k, Q, ldq, tau);
    for (int j = 0; j < k; j++)
        for (int i = 0; i <= j; i++) AT(R, ldr, i, j) = AT(Q, ldq, i, j);
    if (!compact) orgqr(m, k, Q, ldq, tau);
}

static double fro(int m, int ncol, const double *A, int lda) {
    double s = 0.0;
    for (int j = 0; j < ncol; j++)
        for (int i = 0; i < m; i++) s += AT(A, lda, i, j) * AT(A, lda, i, j);
    return sqrt(s);
}

static void copy_mat(int m, int ncol, const double *A, int lda, double *B, int ldb) {
    for (int j = 0; j < ncol; j++) memcpy(&AT(B, ldb, 0, j), &AT(A, lda, 0, j), sizeof(double) * m);
}

/* ------------------------------------------------------------------------------------- */
/* block-GMRES (src/block_gmres.jl:170-411)                                                */
/* ------------------------------------------------------------------------------------- */
typedef struct {
    int memory;
    int restart;
    int reorthogonalization;
    double atol;
    double rtol;
    int itmax;
    double timemax;
    int history;
} orc_gmres_opts;

typedef struct {
    int niter;
    int solved;
    int status;          /* 0 unknown, 1 solved, 2 itmax, 3 time limit */
    double timer;
    int n_residuals;     /* number written into residuals[] */
    int residuals_cap;
    double *residuals;   /* caller-owned */
    int npass;
} orc_stats;

static void push_res(orc_stats *st, double r) {
    if (st->residuals && st->n_residuals < st->residuals_cap) st->residuals[st->n_residuals] = r;
    st->n_residuals++;
}

/* Solve A X = B.  A: CSR n x n.  B, X: n x p column-major.  X0 nullable (warm start; the
 * reference's warm_start! writes a misspelled field, so its X0 path throws -- here X0 works
 * as documented at src/block_gmres.jl:90-103).  M (left) / N (right) preconditioners are
 * applied with ldiv! semantics; kind 0 means the identity (M = I / N = I). */
int orc_block_gmres(int n, const int *rp, const int *ci, const double *av, int p,
                    const double *B, int ldb, double *X, int ldx, const double *X0, int ldx0,
                    int m_kind, const int *m_rp, const int *m_ci, const double *m_v,
                    int n_kind, const int *n_rp, const int *n_ci, const double *n_v,
                    const orc_gmres_opts *o, orc_stats *st) {
    double t0 = now_s();
    orc_prec M = {m_kind, n, m_rp, m_ci, m_v};
    orc_prec N = {n_kind, n, n_rp, n_ci, n_v};
    int MisI = (m_kind == 0), NisI = (n_kind == 0);
    int memory = o->memory;
    if (memory > n / p) memory = n / p;          /* :42 */
    if (memory < 1) memory = 1;
    int restart = o->restart;
    int warm = (X0 != NULL);
    size_t np = (size_t)n * p;
    size_t pp = (size_t)p * p;
    int itmax = o->itmax;
    if (itmax == 0) itmax = 2 * (n / p);          /* :238 */
    /* Without restart the reference grows V/Z/R/H/tau by push! past `memory`
     * (:288-294,357-360); the oracle allocates up front for at most itmax iterations. */
    int cap = restart ? memory : (itmax > memory ? itmax : memory);
    double *W = (double *)malloc(sizeof(double) * np);
    double *Qm = MisI ? NULL : (double *)malloc(sizeof(double) * np);
    double *Pm = NisI ? NULL : (double *)malloc(sizeof(double) * np);
    double *dX = (double *)malloc(sizeof(double) * np);  /* ΔX: warm start / restart accum */
    double *V = (double *)malloc(sizeof(double) * np * (cap + 1));
    double *Z = (double *)malloc(sizeof(double) * pp * (cap + 1));
    double *R = (double *)malloc(sizeof(double) * pp * ((size_t)cap * (cap + 1) / 2));
    double *H = (double *)malloc(sizeof(double) * 2 * pp * cap);
    double *tau = (double *)malloc(sizeof(double) * (size_t)p * (cap + 1));
    double *C = (double *)malloc(sizeof(double) * pp);
    double *D = (double *)malloc(sizeof(double) * 2 * pp);
    double *Ptmp = (double *)malloc(sizeof(double) * pp);
    if (!W || (!MisI && !Qm) || (!NisI && !Pm) || !dX || !V || !Z || !R || !H || !tau || !C ||
        !D || !Ptmp) {
        free(W); free(Qm); free(Pm); free(dX); free(V); free(Z); free(R); free(H); free(tau);
        free(C); free(D); free(Ptmp);
        return ORC_ERR_ALLOC;
    }
    double *Q = MisI ? W : Qm;
    double *R0 = MisI ? W : Qm;
    double *Xr = restart ? dX : X;   /* :204 */
    int p2 = 2 * p;

    st->n_residuals = 0;
    for (int j = 0; j < p; j++) memset(&AT(X, ldx, 0, j), 0, sizeof(double) * n);   /* :216 */
    if (warm) {                                                                      /* :219-222 */
        copy_mat(n, p, X0, ldx0, dX, n);
        for (int j = 0; j < p; j++) memcpy(&AT(W, n, 0, j), &AT(B, ldb, 0, j), sizeof(double) * n);
        orc_spmm(n, rp, ci, av, p, -1.0, dX, n, 1.0, W, n);
        if (restart)
            for (int j = 0; j < p; j++)
                for (int i = 0; i < n; i++) AT(X, ldx, i, j) += dX[(size_t)j * n + i];
    } else {
        copy_mat(n, p, B, ldb, W, n);
    }
    if (!MisI) prec_apply(&M, p, W, n, R0, n);                                       /* :226 */
    double RNorm = fro(n, p, R0, n);
    if (o->history) push_res(st, RNorm);
    double eps = o->atol + o->rtol * RNorm;

    int npass = 0, iter = 0, inner_iter = 0;
    int inner_itmax = itmax;
    int solved = RNorm <= eps;
    int tired = iter >= itmax;
    int overtimed = 0;
    double timemax = o->timemax;

    while (!(solved || tired || overtimed)) {
        int nr = 0;
        memset(V, 0, sizeof(double) * np * (cap + 1));
        memset(R, 0, sizeof(double) * pp * ((size_t)cap * (cap + 1) / 2));
        memset(Z, 0, sizeof(double) * pp * (cap + 1));
        if (restart) {                                                               /* :265-272 */
            memset(Xr, 0, sizeof(double) * np);
            if (npass >= 1) {
                copy_mat(n, p, B, ldb, W, n);
                orc_spmm(n, rp, ci, av, p, -1.0, X, ldx, 1.0, W, n);
                if (!MisI) prec_apply(&M, p, W, n, R0, n);
            }
        }
        memcpy(V, R0, sizeof(double) * np);                                          /* :275-276 */
        orc_householder(n, p, V, n, Z, p, tau, 0);
        npass++;
        inner_iter = 0;
        int inner_tired = 0;
        while (!(solved || inner_tired || overtimed)) {
            inner_iter++;
            int k = inner_iter;
            double *Vk = V + np * (k - 1);
            double *Pk = NisI ? Vk : Pm;
            if (!NisI) prec_apply(&N, p, Vk, n, Pm, n);                              /* :298 */
            orc_spmm(n, rp, ci, av, p, 1.0, Pk, n, 0.0, W, n);                       /* :299 */
            if (!MisI) prec_apply(&M, p, W, n, Q, n);                                /* :300 */
            for (int i = 1; i <= k; i++) {                                           /* :301-304 */
                double *Vi = V + np * (i - 1);
                double *Psi = R + pp * (nr + i - 1);
                gemm(1, p, p, n, 1.0, Vi, n, Q, n, 0.0, Psi, p);
                gemm(0, n, p, p, -1.0, Vi, n, Psi, p, 1.0, Q, n);
            }
            if (o->reorthogonalization) {                                            /* :307-313 */
                for (int i = 1; i <= k; i++) {
                    double *Vi = V + np * (i - 1);
                    double *Psi = R + pp * (nr + i - 1);
                    gemm(1, p, p, n, 1.0, Vi, n, Q, n, 0.0, Ptmp, p);
                    gemm(0, n, p, p, -1.0, Vi, n, Ptmp, p, 1.0, Q, n);
                    for (size_t e = 0; e < pp; e++) Psi[e] += Ptmp[e];
                }
            }
            orc_householder(n, p, Q, n, C, p, tau + (size_t)p * (k - 1), 0);          /* :316 */
            for (int i = 1; i <= k - 1; i++) {                                       /* :320-326 */
                double *Hi = H + 2 * pp * (i - 1);
                double *Ra = R + pp * (nr + i - 1), *Rb = R + pp * (nr + i);
                for (int j = 0; j < p; j++) {
                    memcpy(&AT(D, p2, 0, j), &AT(Ra, p, 0, j), sizeof(double) * p);
                    memcpy(&AT(D, p2, p, j), &AT(Rb, p, 0, j), sizeof(double) * p);
                }
                ormqr_lt(p2, p, Hi, p2, tau + (size_t)p * (i - 1), D, p2, p);
                for (int j = 0; j < p; j++) {
                    memcpy(&AT(Ra, p, 0, j), &AT(D, p2, 0, j), sizeof(double) * p);
                    memcpy(&AT(Rb, p, 0, j), &AT(D, p2, p, j), sizeof(double) * p);
                }
            }
            double *Hk = H + 2 * pp * (k - 1);                                       /* :329-331 */
            double *Rkk = R + pp * (nr + k - 1);
            for (int j = 0; j < p; j++) {
                memcpy(&AT(Hk, p2, 0, j), &AT(Rkk, p, 0, j), sizeof(double) * p);
                memcpy(&AT(Hk, p2, p, j), &AT(C, p, 0, j), sizeof(double) * p);
            }
            double *tk = tau + (size_t)p * (k - 1);
            orc_householder(p2, p, Hk, p2, Rkk, p, tk, 1);
            double *Zk = Z + pp * (k - 1);                                           /* :334-337 */
            for (int j = 0; j < p; j++) {
                memcpy(&AT(D, p2, 0, j), &AT(Zk, p, 0, j), sizeof(double) * p);
                memset(&AT(D, p2, p, j), 0, sizeof(double) * p);
            }
            ormqr_lt(p2, p, Hk, p2, tk, D, p2, p);
            for (int j = 0; j < p; j++) {
                memcpy(&AT(Zk, p, 0, j), &AT(D, p2, 0, j), sizeof(double) * p);
                memcpy(&AT(C, p, 0, j), &AT(D, p2, p, j), sizeof(double) * p);
            }
            RNorm = fro(p, p, C, p);                                                 /* :341-342 */
            if (o->history) push_res(st, RNorm);
            nr += k;
            solved = RNorm <= eps;                                                   /* :349-352 */
            inner_tired = restart ? (k >= (memory < inner_itmax ? memory : inner_itmax))
                                  : (k >= inner_itmax);
            overtimed = (now_s() - t0) > timemax;
            if (!(solved || inner_tired || overtimed)) {                             /* :356-363 */
                memcpy(V + np * k, Q, sizeof(double) * np);
                memcpy(Z + pp * k, C, sizeof(double) * pp);
            }
        }
        /* Block back substitution R Y = Z (:366-375), Y stored in Z. */
        int kk = inner_iter;
        for (int i = kk; i >= 1; i--) {
            int pos = nr + i - kk;
            double *Yi = Z + pp * (i - 1);
            for (int j = kk; j >= i + 1; j--) {
                gemm(0, p, p, p, -1.0, R + pp * (pos - 1), p, Z + pp * (j - 1), p, 1.0, Yi, p);
                pos = pos - j + 1;
            }
            const double *Rii = R + pp * (pos - 1);
            for (int c = 0; c < p; c++) {
                for (int r = p - 1; r >= 0; r--) {
                    double s = AT(Yi, p, r, c);
                    for (int l = r + 1; l < p; l++) s -= AT(Rii, p, r, l) * AT(Yi, p, l, c);
                    AT(Yi, p, r, c) = s / AT(Rii, p, r, r);
                }
            }
        }
        for (int i = 1; i <= kk; i++)                                                /* :378-380 */
            gemm(0, n, p, p, 1.0, V + np * (i - 1), n, Z + pp * (i - 1), p, 1.0, Xr,
                 restart ? n : ldx);
        if (!NisI) {                                                                 /* :381-384 */
            copy_mat(n, p, Xr, restart ? n : ldx, Pm, n);
            prec_apply(&N, p, Pm, n, Xr, restart ? n : ldx);
        }
        if (restart)
            for (int j = 0; j < p; j++)
                for (int i = 0; i < n; i++) AT(X, ldx, i, j) += dX[(size_t)j * n + i];
        inner_itmax -= inner_iter;                                                   /* :388-392 */
        iter += inner_iter;
        tired = iter >= itmax;
        overtimed = (now_s() - t0) > timemax;
    }
    int status = 0;                                                                  /* :397-399 */
    if (tired) status = 2;
    if (solved) status = 1;
    if (overtimed) status = 3;
    if (warm && !restart)                                                            /* :402 */
        for (int j = 0; j < p; j++)
            for (int i = 0; i < n; i++) AT(X, ldx, i, j) += dX[(size_t)j * n + i];
    st->niter = iter;
    st->solved = solved;
    st->status = status;
    st->npass = npass;
    st->timer = now_s() - t0;
    free(W); free(Qm); free(Pm); free(dX); free(V); free(Z); free(R); free(H); free(tau);
    free(C); free(D); free(Ptmp);
    return ORC_OK;
}

/* ------------------------------------------------------------------------------------- */
/* block-BiCGSTAB, CPU variant with LU of K (src/block_bicgstab.jl:70-178)                 */
/* ------------------------------------------------------------------------------------- */

/* LU with partial pivoting (getrf), p x p, in place; piv 0-based.  Returns 0 or i+1 if
 * U(i,i) is exactly zero (Julia's lu! throws SingularException there). */
static int getrf(int p, double *K, int *piv) {
    int info = 0;
    for (int j = 0; j < p; j++) {
        int im = j;
        double mx = fabs(AT(K, p, j, j));
        for (int i = j + 1; i < p; i++)
            if (fabs(AT(K, p, i, j)) > mx) { mx = fabs(AT(K, p, i, j)); im = i; }
        piv[j] = im;
        if (im != j)
            for (int c = 0; c < p; c++) {
                double t = AT(K, p, j, c);
                AT(K, p, j, c) = AT(K, p, im, c);
                AT(K, p, im, c) = t;
            }
        double d = AT(K, p, j, j);
        if (d == 0.0) { if (!info) info = j + 1; continue; }
        for (int i = j + 1; i < p; i++) AT(K, p, i, j) /= d;
        for (int c = j + 1; c < p; c++) {
            double u = AT(K, p, j, c);
            for (int i = j + 1; i < p; i++) AT(K, p, i, c) -= AT(K, p, i, j) * u;
        }
    }
    return info;
}

static void getrs(int p, const double *K, const int *piv, double *Bm, int ncol) {
    for (int c = 0; c < ncol; c++) {
        double *b = Bm + (size_t)c * p;
        for (int j = 0; j < p; j++)
            if (piv[j] != j) { double t = b[j]; b[j] = b[piv[j]]; b[piv[j]] = t; }
        for (int i = 0; i < p; i++)
            for (int l = 0; l < i; l++) b[i] -= AT(K, p, i, l) * b[l];
        for (int i = p - 1; i >= 0; i--) {
            for (int l = i + 1; l < p; l++) b[i] -= AT(K, p, i, l) * b[l];
            b[i] /= AT(K, p, i, i);
        }
    }
}

static double dotm(size_t len, const double *a, const double *b) {
    double s = 0.0;
    for (size_t i = 0; i < len; i++) s += a[i] * b[i];
    return s;
}

/* C nullable: shadow block, defaults to B (:73).  N applied with ldiv semantics (kind 0 = I).
 * Returns ORC_ERR_SINGULAR if the p x p matrix K is exactly singular. */
int orc_block_bicgstab(int n, const int *rp, const int *ci, const double *av, int p,
                       const double *B, int ldb, double *X, int ldx, const double *Cs, int ldc,
                       int n_kind, const int *n_rp, const int *n_ci, const double *n_v,
                       const orc_gmres_opts *o, orc_stats *st) {
    double t0 = now_s();
    orc_prec N = {n_kind, n, n_rp, n_ci, n_v};
    int NisI = (n_kind == 0);
    size_t np = (size_t)n * p, pp = (size_t)p * p;
    if (!Cs) { Cs = B; ldc = ldb; }
    double *Y = (double *)calloc(np, sizeof(double));
    double *P = (double *)malloc(sizeof(double) * np);
    double *R = (double *)malloc(sizeof(double) * np);
    double *V = (double *)calloc(np, sizeof(double));
    double *Q = (double *)calloc(np, sizeof(double));
    double *U = (double *)calloc(np, sizeof(double));
    double *Xc = (double *)calloc(np, sizeof(double));
    double *K = (double *)calloc(pp, sizeof(double));
    double *Dm = (double *)calloc(pp, sizeof(double));
    double *al = (double *)calloc(pp, sizeof(double));
    double *be = (double *)calloc(pp, sizeof(double));
    int *piv = (int *)malloc(sizeof(int) * p);
    int ret = ORC_OK;
    copy_mat(n, p, B, ldb, P, n);                                                    /* :96-98 */
    copy_mat(n, p, B, ldb, R, n);
    double rNorm = fro(n, p, R, n);
    int iter = 0, itmax = o->itmax;
    if (itmax == 0) itmax = 2 * n;                                                   /* :117 */
    st->n_residuals = 0;
    if (o->history) push_res(st, rNorm);
    double eps = o->atol + o->rtol * rNorm;
    int solved = rNorm <= eps, tired = iter >= itmax, overtimed = 0;
    while (!(solved || tired || overtimed)) {
        const double *Yp = P;
        if (!NisI) { prec_apply(&N, p, P, n, Y, n); Yp = Y; }                        /* :134 */
        orc_spmm(n, rp, ci, av, p, 1.0, Yp, n, 0.0, V, n);                           /* :135 */
        gemm(1, p, p, n, 1.0, Cs, ldc, V, n, 0.0, K, p);                             /* :136 */
        gemm(1, p, p, n, 1.0, Cs, ldc, R, n, 0.0, Dm, p);                            /* :137 */
        if (getrf(p, K, piv)) { ret = ORC_ERR_SINGULAR; break; }                     /* :138 */
        memcpy(al, Dm, sizeof(double) * pp);
        getrs(p, K, piv, al, p);                                                     /* :139 */
        memcpy(U, R, sizeof(double) * np);                                           /* :140-141 */
        gemm(0, n, p, p, -1.0, V, n, al, p, 1.0, U, n);
        gemm(0, n, p, p, 1.0, Yp, n, al, p, 0.0, R, n);                              /* :142 */
        for (size_t e = 0; e < np; e++) Xc[e] += R[e];                               /* :143 */
        const double *Yu = U;
        if (!NisI) { prec_apply(&N, p, U, n, Y, n); Yu = Y; }                        /* :144 */
        orc_spmm(n, rp, ci, av, p, 1.0, Yu, n, 0.0, Q, n);                           /* :145 */
        double om = fabs(dotm(np, Q, U)) / fabs(dotm(np, Q, Q));                     /* :146 */
        for (size_t e = 0; e < np; e++) Xc[e] += om * Yu[e];                         /* :147 */
        for (size_t e = 0; e < np; e++) R[e] = U[e] - om * Q[e];                     /* :148 */
        gemm(1, p, p, n, 1.0, Cs, ldc, Q, n, 0.0, Dm, p);                            /* :149 */
        memcpy(be, Dm, sizeof(double) * pp);
        getrs(p, K, piv, be, p);                                                     /* :150 */
        for (size_t e = 0; e < np; e++) U[e] = P[e] - om * V[e];                     /* :151 */
        gemm(0, n, p, p, 1.0, U, n, be, p, 0.0, P, n);                               /* :152 */
        for (size_t e = 0; e < np; e++) P[e] = R[e] - P[e];                          /* :153 */
        iter++;
        rNorm = fro(n, p, R, n);
        if (o->history) push_res(st, rNorm);
        solved = rNorm <= eps;
        tired = iter >= itmax;
        overtimed = (now_s() - t0) > o->timemax;
    }
    copy_mat(n, p, Xc, n, X, ldx);
    int status = 0;
    if (tired) status = 2;
    if (solved) status = 1;
    if (overtimed) status = 3;
    st->niter = iter;
    st->solved = solved;
    st->status = status;
    st->npass = 1;
    st->timer = now_s() - t0;
    free(Y); free(P); free(R); free(V); free(Q); free(U); free(Xc); free(K); free(Dm); free(al);
    free(be); free(piv);
    return ret;
}

/* ------------------------------------------------------------------------------------- */
/* RF oracle: LU with partial pivoting once, then refactor on the fixed pivot order        */
/* (src/cusolverRF.jl:56-220 analysis, :304-314 update!, :317-331 ldiv!).  Dense: used     */
/* only for the small parity cases.                                                        */
/* ------------------------------------------------------------------------------------- */

/* Factor the dense n x n column-major copy of A in place with row pivoting; perm[i] is the
 * original row that ends up in position i.  Returns -(j+1) when |pivot| <= tol * max|A|. */
int orc_lu_factor(int n, double *A, int *perm, double tol) {
    double amax = 0.0;
    for (size_t e = 0; e < (size_t)n * n; e++) amax = fmax(amax, fabs(A[e]));
    for (int i = 0; i < n; i++) perm[i] = i;
    for (int j = 0; j < n; j++) {
        int im = j;
        double mx = fabs(AT(A, n, j, j));
        for (int i = j + 1; i < n; i++)
            if (fabs(AT(A, n, i, j)) > mx) { mx = fabs(AT(A, n, i, j)); im = i; }
        if (mx <= tol * amax) return -(j + 1);
        if (im != j) {
            for (int c = 0; c < n; c++) {
                double t = AT(A, n, j, c);
                AT(A, n, j, c) = AT(A, n, im, c);
                AT(A, n, im, c) = t;
            }
            int t = perm[j]; perm[j] = perm[im]; perm[im] = t;
        }
        double d = AT(A, n, j, j);
        for (int i = j + 1; i < n; i++) AT(A, n, i, j) /= d;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (n > 256)
        for (int c = j + 1; c < n; c++) {
            double u = AT(A, n, j, c);
            if (u != 0.0)
                for (int i = j + 1; i < n; i++) AT(A, n, i, c) -= AT(A, n, i, j) * u;
        }
    }
    return 0;
}

/* Refactor: rows already permuted by perm, no pivoting (the RF refactor keeps P and Q). */
int orc_lu_refactor(int n, double *A, const int *perm_unused) {
    (void)perm_unused;
    for (int j = 0; j < n; j++) {
        double d = AT(A, n, j, j);
        if (d == 0.0) return -(j + 1);
        for (int i = j + 1; i < n; i++) AT(A, n, i, j) /= d;
#pragma omp parallel for num_threads(g_threads) schedule(static) if (n > 256)
        for (int c = j + 1; c < n; c++) {
            double u = AT(A, n, j, c);
            if (u != 0.0)
                for (int i = j + 1; i < n; i++) AT(A, n, i, c) -= AT(A, n, i, j) * u;
        }
    }
    return 0;
}

/* Solve with the factored, row-permuted LU: X (n x nrhs, col-major) overwritten. */
void orc_lu_solve(int n, const double *LU, const int *perm, int nrhs, double *X, int ldx) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int c = 0; c < nrhs; c++) {
        double *x = X + (size_t)c * ldx;
        double *y = (double *)malloc(sizeof(double) * n);
        for (int i = 0; i < n; i++) y[i] = x[perm[i]];
        for (int i = 0; i < n; i++)
            for (int l = 0; l < i; l++) y[i] -= AT(LU, n, i, l) * y[l];
        for (int i = n - 1; i >= 0; i--) {
            for (int l = i + 1; l < n; l++) y[i] -= AT(LU, n, i, l) * y[l];
            y[i] /= AT(LU, n, i, i);
        }
        memcpy(x, y, sizeof(double) * n);
        free(y);
    }
}
