/*
 * bpf.h -- C ABI of libbpf.so, the B200 (sm_100a) multi-RHS sparse solve library.
 *
 * Each entry point replaces one call of exanauts/BlockPowerFlow.jl (Julia) that a host
 * binding (ccall from Julia, ctypes from Python) forwards here.  The reference interface each
 * one stands in for is cited beside it as `file:line` of that project.
 *
 * Conventions
 *  - Every function returns a bpf_status; on failure bpf_last_error(ctx) says why.
 *  - Dense blocks (B, X, Y, ...) are DEVICE pointers to column-major n x p matrices with an
 *    explicit leading dimension (Julia's CuMatrix{Float64}).  Internal layouts are private.
 *  - CSR descriptors hold DEVICE pointers and are borrowed: the library never frees them.
 *    index_base 1 accepts CUDA.jl's 1-based CuSparseMatrixCSR arrays as they are.
 *  - All work is ordered on the context's stream.  A call returns only after the stream has
 *    finished when it has to hand host scalars back (solver statistics); the others are
 *    asynchronous with respect to the host.
 *  - A context is not thread-safe: use one per host thread / Julia task.
 */
#ifndef BPF_H_
#define BPF_H_

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BPF_API __attribute__((visibility("default")))
#else
#define BPF_API
#endif

typedef enum {
    BPF_SUCCESS = 0,
    BPF_ERR_INVALID_VALUE = 1,  /* bad argument (null pointer, negative size, ...)        */
    BPF_ERR_DIMENSION = 2,      /* "System must be square" / "Inconsistent problem size" */
    BPF_ERR_CUDA = 3,           /* a CUDA runtime call failed                            */
    BPF_ERR_ALLOC = 4,          /* device or host allocation failed                      */
    BPF_ERR_SINGULAR = 5,       /* zero / non-positive pivot in a factorization           */
    BPF_ERR_NOT_SUPPORTED = 6,  /* option combination the reference rejects as well      */
    BPF_ERR_TIMEOUT = 7,        /* a bounded device-side wait gave up                    */
    BPF_ERR_NUMERIC = 8         /* NaN/Inf met where the algorithm cannot continue       */
} bpf_status;

typedef enum { BPF_F64 = 0, BPF_F32 = 1 } bpf_dtype;

/* Termination status of a Krylov solve; bpf_solve_status_string gives the reference's text
 * (src/block_gmres.jl:397-399, src/block_bicgstab.jl:160-171). */
typedef enum {
    BPF_SOLVE_UNKNOWN = 0,
    BPF_SOLVE_SOLVED = 1,       /* "solution good enough given atol and rtol" */
    BPF_SOLVE_ITMAX = 2,        /* "maximum number of iterations exceeded"    */
    BPF_SOLVE_TIMEMAX = 3       /* "time limit exceeded"                      */
} bpf_solve_status;

/* Fill-reducing orderings of the RF analysis (src/cusolverRF.jl:70-95). */
typedef enum {
    BPF_ORDER_AMD = 0,      /* :AMD   (reference default)                          */
    BPF_ORDER_MDQ = 1,      /* :MDQ   minimum degree on the quotient graph          */
    BPF_ORDER_METIS = 2,    /* :METIS nested dissection                             */
    BPF_ORDER_RCM = 3,      /* :RCM   reverse Cuthill-McKee                          */
    BPF_ORDER_NATURAL = 4   /* no reordering                                         */
} bpf_ordering;

/* Arithmetic of the preconditioner's triangular factors.  BPF_F32 keeps an FP32 copy of the
 * factors and runs the triangular solves in FP32 (FP64 in / FP64 out). */
typedef bpf_dtype bpf_factor_dtype;

typedef struct bpf_ctx bpf_ctx;
typedef struct bpf_prec bpf_prec;
typedef struct bpf_rf bpf_rf;

/* CuSparseMatrixCSR{Float64,Cint}: n x n, device arrays, borrowed. */
typedef struct {
    int n;
    int nnz;
    const int *rowptr;   /* n+1 */
    const int *colind;   /* nnz, sorted within each row */
    const void *vals;    /* nnz, dtype below */
    int index_base;      /* 0 or 1 */
    int dtype;           /* bpf_dtype; only BPF_F64 for the system matrix */
} bpf_csr_desc;

/* Keyword arguments of block_gmres (src/block_gmres.jl:142-145). */
typedef struct {
    int memory;              /* default 20 */
    int restart;             /* bool */
    int reorthogonalization; /* bool */
    int ldiv;                /* bool: preconditioners applied with ldiv! (true) or mul! */
    double atol;             /* default sqrt(eps) */
    double rtol;             /* default sqrt(eps) */
    int itmax;               /* 0 -> 2*div(n,p) */
    double timemax;          /* seconds, <= 0 or inf -> no limit */
    int verbose;             /* print every `verbose` iterations (host stdout) */
    int history;             /* bool: record residual norms */
} bpf_gmres_opts;

/* Keyword arguments of block_bicgstab (src/block_bicgstab.jl:182-185). */
typedef struct {
    double atol;
    double rtol;
    int itmax;               /* 0 -> 2n */
    double timemax;
    int verbose;
    int history;
} bpf_bicgstab_opts;

/* BlockGMRESStats / SimpleStats (src/block_utils.jl:62-68, src/block_bicgstab.jl:15-21). */
typedef struct {
    int niter;
    int solved;              /* bool */
    int status;              /* bpf_solve_status */
    double timer;            /* seconds */
    int n_residuals;         /* residual norms produced (may exceed the capacity) */
    int residuals_capacity;  /* capacity of `residuals` */
    double *residuals;       /* caller-owned HOST buffer or NULL */
    int npass;               /* restart passes (GMRES) */
} bpf_stats;

/* ---- context ------------------------------------------------------------------------- */
/* stream: a cudaStream_t (NULL = legacy default stream).  Replaces the implicit CUDA.jl
 * task-local stream / library handles of src/BlockPowerFlow.jl:1-31. */
BPF_API bpf_status bpf_ctx_create(bpf_ctx **ctx, void *stream);
BPF_API bpf_status bpf_ctx_set_stream(bpf_ctx *ctx, void *stream);
BPF_API bpf_status bpf_ctx_destroy(bpf_ctx *ctx);
BPF_API const char *bpf_last_error(const bpf_ctx *ctx);
BPF_API const char *bpf_solve_status_string(int status);
/* Number of kernels this library launched on the context (a running counter). */
BPF_API long long bpf_ctx_kernel_launches(const bpf_ctx *ctx);

/* Failure detection.  Every cross-block wait of the library's kernels (the grid barriers of the
 * cooperative triangular solves and factorizations) gives up after a bounded number of polls,
 * records the timeout and returns, so a block that never arrives ends the call with
 * BPF_ERR_TIMEOUT and leaves the context usable.  No counterpart in the reference, whose
 * library calls block until the device finishes.  polls = 0 restores the default (~2^21 polls,
 * about a second); smaller limits shorten the watchdog. */
BPF_API bpf_status bpf_ctx_set_wait_limit(bpf_ctx *ctx, long long polls);
/* Self-test of that path: a cooperative launch of nblocks (2.. co-resident maximum) blocks that
 * meet at one grid barrier, block absent_block (-1: none) skipping it.  Returns BPF_SUCCESS when
 * every block passed, BPF_ERR_TIMEOUT when the others gave up waiting for the absent one;
 * *arrived (host, nullable) = the blocks that passed the barrier. */
BPF_API bpf_status bpf_selftest_grid_barrier(bpf_ctx *ctx, int nblocks, int absent_block, int *arrived);

/* Per-kernel-class device timing (CUDA events recorded around each launch on the context's
 * stream).  No counterpart in the reference: it stands in for the CUDA.@time / @time
 * measurements of test/*.jl and is what the benchmark uses to put a launch-averaged kernel
 * duration next to its roofline.  bpf_ctx_set_timing(ctx, 1) clears and starts recording. */
typedef enum {
    BPF_KC_SPMM = 0,    /* CSR SpMM                                   */
    BPF_KC_TRSV = 1,    /* preconditioner / RF triangular solves      */
    BPF_KC_FACTOR = 2,  /* ILU0 / IC0 / RF numeric factorization      */
    BPF_KC_GRAM = 3,    /* block Gram products (split over rows)      */
    BPF_KC_TSMM = 4,    /* tall x small block products                */
    BPF_KC_SMALL = 5,   /* other one-CTA p x p kernels (BiCGSTAB solves) */
    BPF_KC_CHOL = 6,    /* Cholesky-QR: Cholesky + inverse of p x p Gram */
    BPF_KC_HESS = 7,    /* block Hessenberg QR update (apply + factor) */
    BPF_KC_BACKSUB = 8, /* block back substitution of block-GMRES     */
    BPF_KC_MLP = 9,     /* learned warm start: tensor-core GEMMs       */
    BPF_KC_BATCH = 10,  /* batched solve: the persistent solve kernel (its ILU(0) kernel counts as FACTOR) */
    BPF_KC_PF = 11,     /* power-flow mismatch and Jacobian assembly  */
    BPF_KC_COUNT = 12
} bpf_kernel_class;
BPF_API bpf_status bpf_ctx_set_timing(bpf_ctx *ctx, int on);
/* Totals since bpf_ctx_set_timing(ctx, 1): device milliseconds, launches, and the launches'
 * algorithmic DRAM bytes and flops (the roofline numerators; each kernel's formula is stated
 * beside it in the sources).  Any output pointer may be NULL. */
BPF_API bpf_status bpf_ctx_kernel_time(bpf_ctx *ctx, int kernel_class, double *total_ms,
                                       long long *launches, double *bytes, double *flops);

/* ---- tensor-core GEMM of the learned warm start ------------------------------------------
 * D (M x N, FP32, row stride ldd) = [D +] A (M x K) B (N x K)^T with A and B row-major BF16
 * (K contiguous; lda, ldb multiples of 8; K a multiple of 64), on the tcgen05 tensor cores
 * with the accumulator in TMEM; splits = K slices (0: chosen to fill the GPU).  No counterpart
 * in the reference (whose solvers have no learned part); the building block of bpf_mlp_*. */
BPF_API bpf_status bpf_tc_gemm_bf16(bpf_ctx *ctx, int M, int N, int K, const void *A, int lda,
                                    const void *B, int ldb, float *D, int ldd, int accumulate,
                                    int splits);

/* ---- learned warm start and deflation basis -----------------------------------------------
 * No counterpart in the reference: a 3-layer MLP (n -> hidden -> hidden -> n, LeakyReLU 0.25,
 * BF16 weights with FP32 masters, tensor-core products, Adam) that maps a right-hand side b to
 * a warm start x0 = s ||b|| f(b / ||b||) for block-GMRES and spans a low-rank deflation basis.
 * It is trained on the solver's own (b, x) pairs; the solver then runs from x0 to the requested
 * residual, so a poor network costs iterations, never accuracy.  All pointers are device
 * pointers, blocks column-major; batches of at most 128 columns for the training calls. */
typedef struct bpf_mlp bpf_mlp;
BPF_API bpf_status bpf_mlp_create(bpf_ctx *ctx, int n, int hidden, unsigned long long seed,
                                  bpf_mlp **mlp);
BPF_API bpf_status bpf_mlp_destroy(bpf_mlp *mlp);
/* s: the output scale (the training set's typical ||x|| / ||b||). */
BPF_API bpf_status bpf_mlp_set_scale(bpf_mlp *mlp, double scale);
/* X (n x p) = warm starts for the columns of B (n x p), any p. */
BPF_API bpf_status bpf_mlp_forward(bpf_mlp *mlp, int p, const double *B, int ldb, double *X,
                                   int ldx);
/* Loss L = (1/p) sum_j ||y_j - t_j||^2 / ||t_j||^2 (t_j = x_j / (s ||b_j||)) of the batch
 * (B, X), p <= 128, and its gradients in the parameters' gradient buffers (bpf_mlp_params);
 * *loss (host, nullable) receives L. */
BPF_API bpf_status bpf_mlp_gradients(bpf_mlp *mlp, int p, const double *B, int ldb,
                                     const double *X, int ldx, double *loss);
/* bpf_mlp_gradients followed by one Adam step (beta 0.9 / 0.999) with learning rate lr. */
BPF_API bpf_status bpf_mlp_train_step(bpf_mlp *mlp, int p, const double *B, int ldb,
                                      const double *X, int ldx, double lr, double *loss);
/* Device FP32 parameter `which` (0 W1 [hidden x np], 1 b1, 2 W2 [hidden x hidden], 3 b2,
 * 4 W3 [np x hidden], 5 b3 [np]; np = n rounded up to 128, padding zero), its gradient buffer
 * and shape.  After writing parameters, call bpf_mlp_refresh. */
BPF_API bpf_status bpf_mlp_params(bpf_mlp *mlp, int which, float **w, float **grad,
                                  long long *rows, long long *cols);
BPF_API bpf_status bpf_mlp_refresh(bpf_mlp *mlp);
/* Copy parameter `which` (or its gradient, grad = 1) to the device buffer buf (to_network = 0)
 * or from it into the network (to_network = 1; refreshes the BF16 copies). */
BPF_API bpf_status bpf_mlp_param_copy(bpf_mlp *mlp, int which, int grad, float *buf,
                                      int to_network);
/* Z (n x rank) = an orthonormal basis of the network's outputs on rank seeded Gaussian
 * probes (the span it has learned), for deflated block-GMRES. */
BPF_API bpf_status bpf_mlp_basis(bpf_mlp *mlp, int rank, unsigned long long seed, double *Z,
                                 int ldz);

/* ---- sparse x dense block -------------------------------------------------------------- */
/* Y = alpha*A*X + beta*Y: mul!(W, A, P) of src/block_gmres.jl:299 (CSR SpMM). */
BPF_API bpf_status bpf_spmm(bpf_ctx *ctx, const bpf_csr_desc *A, int p, double alpha,
                            const double *X, int ldx, double beta, double *Y, int ldy);

/* Reduced QR of an n x p block, Q overwritten by the orthonormal factor and R (p x p, upper,
 * ldr) written: householder!(Q, R, tau) of src/block_utils.jl:46-53.  Computed as shifted /
 * plain Cholesky-QR2, so R's diagonal is positive (LAPACK's may be negative; Q and R differ from
 * LAPACK's by the same diagonal +-1 scaling). */
BPF_API bpf_status bpf_householder(bpf_ctx *ctx, int n, int p, double *Q, int ldq, double *R,
                                   int ldr);
/* householder(A; compact) with LAPACK's conventions, src/block_utils.jl:38-53 (geqrf, then
 * orgqr unless compact): R (p x p, ldr) has the signs geqrf gives (R_jj = -sign(alpha_j) ||x_j||),
 * tau (device, p doubles, nullable) the reflectors' scalars; Q is overwritten by orgqr's
 * orthonormal factor (compact = 0) or by geqrf's compact form (compact = 1: R on and above the
 * diagonal, the unit-lower reflector vectors below it).  Computed from Cholesky-QR2 by Householder
 * reconstruction (the LU of Q - S with LAPACK's sign choice), so Q, R and tau equal LAPACK's up
 * to rounding. */
BPF_API bpf_status bpf_householder_lapack(bpf_ctx *ctx, int n, int p, double *Q, int ldq, double *R,
                                          int ldr, double *tau, int compact);

/* ---- preconditioners ------------------------------------------------------------------- */
/* ilu0(A, nrhs) -- src/preconditioners_nvidia.jl:42-47 (csrilu02 on A's pattern). */
BPF_API bpf_status bpf_ilu0_create(bpf_ctx *ctx, const bpf_csr_desc *A, int nrhs,
                                   int factor_dtype, bpf_prec **prec);
/* ic0(A, nrhs) -- src/preconditioners_nvidia.jl:6-11 (csric02 on A's lower triangle). */
BPF_API bpf_status bpf_ic0_create(bpf_ctx *ctx, const bpf_csr_desc *A, int nrhs,
                                  int factor_dtype, bpf_prec **prec);

/* ilu0 / ic0 with a symmetric reordering of the pattern: the factors are those of
 * A(perm, perm), and bpf_prec_apply keeps ldiv! semantics in A's own ordering (y = M \ x with
 * M = P' L U P).  No counterpart in the reference, whose ilu0 / ic0 factor A in its natural
 * order (src/preconditioners_nvidia.jl:6-11,42-47); the orderings are those of the RF analysis
 * (src/cusolverRF.jl:70-95): BPF_ORDER_RCM (reverse Cuthill-McKee), BPF_ORDER_AMD / MDQ
 * (minimum degree), BPF_ORDER_NATURAL (same as bpf_ilu0_create); BPF_ORDER_METIS is not
 * available.  nrhs sizes the factor-ordered scratch of the solves (grown on demand by
 * bpf_prec_apply and the Krylov solvers; bpf_prec_apply_noalloc uses it as it is). */
BPF_API bpf_status bpf_ilu0_create_ordered(bpf_ctx *ctx, const bpf_csr_desc *A, int nrhs,
                                           int factor_dtype, int ordering, bpf_prec **prec);
BPF_API bpf_status bpf_ic0_create_ordered(bpf_ctx *ctx, const bpf_csr_desc *A, int nrhs,
                                          int factor_dtype, int ordering, bpf_prec **prec);
/* The preconditioner's ordering: perm[i] = the row of A that is row i of the factors (the
 * identity for a natural-order preconditioner); perm is a host array of n ints. */
BPF_API bpf_status bpf_prec_permutation(const bpf_prec *P, int *perm);
/* New values on the same pattern (device pointer, nnz doubles), then refactor.  The
 * reference rebuilds the preconditioner with ilu0(A) after each Jacobian update
 * (benchmarks/benchmarks_nvidia.jl:44). */
BPF_API bpf_status bpf_prec_refactor(bpf_prec *prec, const double *vals);
/* ldiv!(Y, P, X): Y = U \ (L \ X) (ILU0) or Y = L' \ (L \ X) (IC0);
 * src/preconditioners_nvidia.jl:13-35,49-71.  Y may equal X. */
BPF_API bpf_status bpf_prec_apply(bpf_prec *prec, int p, const double *X, int ldx, double *Y,
                                  int ldy);
/* No counterpart in the reference.  The same Y = P \ X as bpf_prec_apply for callers that
 * cannot allocate device memory once the preconditioner exists: hosts whose device memory
 * belongs to an external pool or a fixed start-up arena (a cudaMalloc behind the pool's back can
 * fail or fragment it) and real-time loops that forbid allocation after set-up (a cudaMalloc
 * synchronizes the device and takes an unbounded time).  Its scratch is a static 8 MiB device
 * array instead of a cudaMalloc'd workspace.  Limit: n * min(p, 256) <= 1,048,576 doubles, else
 * BPF_ERR_NOT_SUPPORTED; a reordered preconditioner also takes at most the nrhs it was created
 * for per 256-column slice (its own scratch is never grown here).  All calls on a device share
 * the array and it keeps the last call's contents (calls that overlap on the GPU race); the
 * first call on a device after a context was created there looks the array's address up. */
BPF_API bpf_status bpf_prec_apply_noalloc(bpf_prec *prec, int p, const double *X, int ldx,
                                          double *Y, int ldy);
/* Copy the factor values (A's pattern, nnz doubles, device pointer) out: the P field of
 * NVIDIA_ILU0 / NVIDIA_IC0 (src/preconditioners_nvidia.jl:1-4,37-40). */
BPF_API bpf_status bpf_prec_factor_values(const bpf_prec *prec, double *vals);
/* Number of dependency levels of the forward (L) and backward (U or L') solves. */
BPF_API bpf_status bpf_prec_levels(const bpf_prec *prec, int *levels_lower, int *levels_upper);
BPF_API bpf_status bpf_prec_destroy(bpf_prec *prec);

/* Block-Jacobi preconditioner (ExaPF's LinearSolvers.BlockJacobiPreconditioner, used by
 * test/block_gmres.jl:5,17,22 and benchmarks/benchmarks_nvidia.jl:47-51; ExaPF is not part of the
 * reference): the dense inverses of the diagonal blocks of A, applied by multiplication, y = P x
 * (mul! semantics: bpf_prec_apply multiplies; block_gmres takes it with ldiv = false).  Blocks are
 * consecutive runs of block_size (1..32) rows in `ordering` (BPF_ORDER_NATURAL, _RCM, _AMD or
 * _MDQ; ExaPF's METIS partition is not available: _METIS returns BPF_ERR_NOT_SUPPORTED).
 * bpf_prec_refactor recomputes the inverses from new values; a singular block returns
 * BPF_ERR_SINGULAR. */
BPF_API bpf_status bpf_block_jacobi_create(bpf_ctx *ctx, const bpf_csr_desc *A, int block_size,
                                           int ordering, bpf_prec **prec);

/* ---- block Krylov solvers -------------------------------------------------------------- */
/* block_gmres(A, B[, X0]; kwargs...) -> (X, stats): src/block_gmres.jl:127-154,170-411.
 * X0 nullable (warm start).  M: left, N: right preconditioner, either nullable (= I).
 * p > 128: solved in column slices of at most 128, each by block-GMRES with atol scaled by
 * sqrt(p_slice / p), so the whole block still meets ||R||_F <= atol + rtol ||B||_F; stats give
 * the largest slice iteration count and the root-sum-square residual history. */
BPF_API bpf_status bpf_block_gmres(bpf_ctx *ctx, const bpf_csr_desc *A, int p,
                                   const double *B, int ldb, double *X, int ldx,
                                   const double *X0, int ldx0, const bpf_prec *M,
                                   const bpf_prec *N, const bpf_gmres_opts *opts,
                                   bpf_stats *stats);
/* block_gmres with a deflation basis Z (n x rank device block, column-major, rank <= p): the
 * GCRO form of Krylov-subspace augmentation -- Q_C = orthonormalized A Z, the starting residual
 * projected off Q_C, every new block orthogonalized against Q_C before the basis, and
 * x = x0 + Z R^{-1} Q_C^T r0 + N \ V y - Z R^{-1} E y.  Same options, stopping rule (epsilon from
 * the unprojected initial residual) and statistics as bpf_block_gmres; right preconditioning
 * only.  No counterpart in the reference: the learned deflation basis of bpf_mlp_basis is its
 * intended input (any basis works; the solver still reaches the requested residual). */
BPF_API bpf_status bpf_block_gmres_deflated(bpf_ctx *ctx, const bpf_csr_desc *A, int p,
                                            const double *B, int ldb, double *X, int ldx,
                                            const double *X0, int ldx0, const bpf_prec *M,
                                            const bpf_prec *N, const bpf_gmres_opts *opts,
                                            const double *Z, int ldz, int rank, bpf_stats *stats);

/* block_bicgstab(A, B; C=B, N, kwargs...) -> (X, stats): src/block_bicgstab.jl:182-299.
 * C (shadow block) nullable -> B.  N: right preconditioner (nullable = I), applied as
 * Y = N^{-1} P exactly as the reference's comment at :247 states. */
BPF_API bpf_status bpf_block_bicgstab(bpf_ctx *ctx, const bpf_csr_desc *A, int p,
                                      const double *B, int ldb, double *X, int ldx,
                                      const double *C, int ldc, const bpf_prec *N,
                                      const bpf_bicgstab_opts *opts, bpf_stats *stats);

/* ---- batched block-GMRES ----------------------------------------------------------------
 * Many independent systems, each with its own Jacobian and right-hand-side block, solved by
 * ILU(0)-preconditioned block-GMRES in one CUDA-graph launch: the ILU(0) of every system, then
 * ONE persistent kernel in which each CTA takes work units (a system and a slice of <= 32 of its
 * right-hand-side columns) from a queue, longest first.  No counterpart in the reference, whose
 * solvers take one system per call; each unit follows block_gmres (src/block_gmres.jl:170-411)
 * with a right ILU(0) (src/preconditioners_nvidia.jl:42-71), unrestarted while its basis lasts.
 * Stopping test per unit: ||R_slice||_F <= atol + rtol ||B_slice||_F (so the whole block meets
 * ||R||_F <= rtol ||B||_F when atol = 0). */
typedef struct bpf_batch bpf_batch;
typedef struct {
    double atol;        /* default 0 */
    double rtol;        /* default 1e-8 */
    int itmax;          /* iterations per unit; 0 -> max(2 div(n, q), 50) */
    int memory;         /* basis blocks per unit; 0 -> sized from n and q (restart when full) */
    int factor_dtype;   /* BPF_F32 (default: FP32 factors, flexible FP64 outer) or BPF_F64 */
    int ordering;       /* BPF_ORDER_AMD (default, minimum degree), _MDQ, _RCM or _NATURAL */
    int slice;          /* widest column slice q, 1..32; 0 -> 16 */
    int ctas_per_sm;    /* resident solve CTAs per SM asked for, 1 or 2 (0 -> 2); the solve
                           kernel holds 255 registers per thread, so one CTA per SM runs */
} bpf_batch_opts;
BPF_API void bpf_batch_opts_default(bpf_batch_opts *opts);
/* Analyse nsys systems (A[s]: device CSR, FP64; nrhs[s] >= 1 columns) and capture the solve
 * graph.  A[s].vals is re-read by every solve: new values on the same pattern go in place. */
BPF_API bpf_status bpf_batch_plan(bpf_ctx *ctx, int nsys, const bpf_csr_desc *A, const int *nrhs,
                                  const bpf_batch_opts *opts, bpf_batch **batch);
/* bpf_batch_plan with a widest column slice per system: slices[s] in 1..32, or 0 for
 * opts->slice (slices NULL: opts->slice for every system).  Narrower slices for the systems
 * whose units take longest shorten the critical path of the persistent solve (its makespan is
 * at least its longest unit). */
BPF_API bpf_status bpf_batch_plan_sliced(bpf_ctx *ctx, int nsys, const bpf_csr_desc *A,
                                         const int *nrhs, const int *slices,
                                         const bpf_batch_opts *opts, bpf_batch **batch);
/* X[s] (n_s x nrhs[s], column-major, ld ldx[s]) = A[s] \ B[s] for every s; B, X, ldb, ldx are
 * HOST arrays of nsys entries (device block pointers; ldb / ldx NULL -> n_s).  stats (nsys
 * entries, nullable): niter = the most iterations of the system's units, solved = all units
 * met the tolerance, npass = most restart cycles.  BPF_ERR_SINGULAR names the first system whose
 * ILU(0) met a zero pivot (the other systems are still solved).  Synchronizes the context's
 * stream; one solve of a plan at a time (its unit workspaces and IO table are shared). */
BPF_API bpf_status bpf_batch_solve(bpf_batch *batch, const double *const *B, const int *ldb,
                                   double *const *X, const int *ldx, bpf_stats *stats);
/* Per unit of the last solve (arrays of bpf_batch_info's nunits entries, each nullable). */
BPF_API bpf_status bpf_batch_unit_stats(const bpf_batch *batch, int *sys, int *col0, int *q,
                                        int *memory, int *niter, int *status, double *rnorm0,
                                        double *rnorm);
/* SM cycles of each unit of the last solve by phase: 8 entries per unit (triangular solves,
 * SpMM, Gram products, block updates, Cholesky-QR, Hessenberg update, back substitution, and
 * the unit's total), counted by thread 0 of the unit's CTA. */
BPF_API bpf_status bpf_batch_unit_cycles(const bpf_batch *batch, long long *cycles);
BPF_API bpf_status bpf_batch_info(const bpf_batch *batch, int *nunits, int *grid,
                                  long long *device_bytes);
BPF_API bpf_status bpf_batch_destroy(bpf_batch *batch);

/* ---- power-flow assembly (the caller of the solve path) --------------------------------
 * The Newton power-flow loop whose linear systems the path solves: the mismatch
 * F(x) = S(V(x)) - S_spec, S = V conj(Ybus V), the Jacobian Gx = dF/dx on a fixed pattern and the
 * control Jacobian Gu = dF/du, assembled on the device.  The reference's benchmark reads Gx and Gu
 * that ExaPF assembled (benchmarks/benchmarks_nvidia.jl:29-39) and refactors Gx once per Newton
 * step (src/cusolverRF.jl:304-314).  Unknowns x = [theta(non-slack buses); |V|(PQ buses)] and
 * equations F = [P(non-slack); Q(PQ)], both in bus order; controls u = |V| of the slack bus, then
 * of the PV buses in bus order (Gu: n x n_ctrl).  An object holds the bus voltages of its last
 * evaluation and its norm word: one call at a time per object (its context's stream orders them). */
typedef struct bpf_pf bpf_pf;
/* Ybus: HOST CSR, 0-based, n_bus rows, sorted unique columns, vals interleaved (re, im).
 * bus_type: 1 PQ, 2 PV, 3 slack (exactly one).  vm_fixed / va_fixed (n_bus): |V| and angle at
 * the buses where they are not unknowns; s_spec: 2 n_bus doubles (P, Q) interleaved.  jac: the
 * device pattern of Gx (0- or 1-based); every entry the buses' coupling produces must be in it
 * (BPF_ERR_INVALID_VALUE names the first missing one), other entries are written as zeros. */
BPF_API bpf_status bpf_pf_create(bpf_ctx *ctx, int n_bus, const int *ybus_rowptr, const int *ybus_colind,
                                 const double *ybus_vals, const int *bus_type, const double *vm_fixed,
                                 const double *va_fixed, const double *s_spec, const bpf_csr_desc *jac,
                                 bpf_pf **pf);
BPF_API bpf_status bpf_pf_info(const bpf_pf *pf, int *n, int *n_ctrl, int *n_bus);
/* F (device, n) = mismatch at x + alpha dx (dx nullable -> at x); x_out (nullable, may alias x)
 * receives that point.  norm_inf (host, nullable): max |F|, NaN if any entry is; when given, the
 * call synchronizes the context's stream. */
BPF_API bpf_status bpf_pf_mismatch(bpf_pf *pf, const double *x, const double *dx, double alpha,
                                   double *x_out, double *F, double *norm_inf);
/* Gx values at x into jac_vals (device, the pattern's nnz, CSR order); gu (nullable, device,
 * column-major n x n_ctrl, ld ldgu >= n) = Gu at x. */
BPF_API bpf_status bpf_pf_jacobian(bpf_pf *pf, const double *x, double *jac_vals, double *gu, int ldgu);
BPF_API bpf_status bpf_pf_destroy(bpf_pf *pf);

/* ---- refactorization (cusolverRF replacement) ------------------------------------------ */
/* CusolverRfLU(A; ordering, tol, fast_mode) / CusolverRfLUBatch(A, batch; ...):
 * src/cusolverRF.jl:222-301,336-419.  Host analysis (ordering + threshold-pivoted LU), then
 * the device refactor.  batch >= 1 (1 = CusolverRfLU).  A zero pivot (|pivot| <= tol *
 * max|A|) returns BPF_ERR_SINGULAR; the reference constructs a SingularException there but
 * never throws it (:164-166). */
BPF_API bpf_status bpf_rf_analyze(bpf_ctx *ctx, const bpf_csr_desc *A, int ordering,
                                  double tol, int fast_mode, int batch, bpf_rf **rf);
/* update!(rflu, A) / lu!(rflu, A): new values on A's pattern (device, nnz doubles), then the
 * device refactor (src/cusolverRF.jl:304-314,334,422-434). */
BPF_API bpf_status bpf_rf_refactor(bpf_rf *rf, const double *vals);
/* rf_batch_refactor!(rflu, Anzval): replica r takes column r of the nnz x batch matrix
 * `vals` (leading dimension ld) (src/cusolverRF.jl:472-481). */
BPF_API bpf_status bpf_rf_refactor_batch(bpf_rf *rf, const double *vals, int ld);
/* ldiv!(x, rflu, b) / ldiv!(rflu, x) / solve! (src/cusolverRF.jl:317-331,439-470): in place,
 * X is n x nrhs (ldx).  Single mode solves every column with the one factorization
 * (multi-RHS; the reference allows only nrhs = 1, :228-230).  Batch mode requires
 * nrhs == batch and solves column r with replica r. */
BPF_API bpf_status bpf_rf_solve(bpf_rf *rf, int nrhs, double *X, int ldx);
/* X = A \ B by the refactored LU followed by `steps` rounds of iterative refinement
 * (X += LU \ (B - A X), residual in FP64 with A's current values: the matrix given to the last
 * bpf_rf_refactor, as a device CSR descriptor).  No counterpart in the reference, whose
 * cusolverRf solve (src/cusolverRF.jl:317-331) applies the refactored LU once; a refactorization
 * that keeps the analysis's pivot order on new values can lose a digit or two to growth, and one
 * round recovers them.  B and X are distinct column-major blocks; uniform factors only. */
BPF_API bpf_status bpf_rf_solve_refined(bpf_rf *rf, const bpf_csr_desc *A, int nrhs, const double *B,
                                        int ldb, double *X, int ldx, int steps);
/* nnz of L (strict lower) and U (incl. diagonal), and the host-side P/Q permutations
 * (0-based, n ints each; nullable). */
BPF_API bpf_status bpf_rf_info(const bpf_rf *rf, int *nnzL, int *nnzU, int *P, int *Q);
/* cudestroy!(rflu) (src/cusolverRF.jl:17-22,54). */
BPF_API bpf_status bpf_rf_destroy(bpf_rf *rf);

#ifdef __cplusplus
}
#endif

#endif /* BPF_H_ */
