// Sparse LU refactorization on a fixed pattern: the cusolverRF replacement
// (src/cusolverRF.jl: CusolverRfLU :222-301, update! :304-314, ldiv! :317-331,
//  CusolverRfLUBatch :336-419, batch update!/solve!/ldiv! :422-470, rf_batch_refactor! :472-481).
//
// Host analysis (once per pattern, as in the reference, which runs cusolverSp's host LU):
//   1. fill-reducing symmetric ordering q of A + A^T: minimum degree on the elimination graph
//      (Tinney-Walker / George-Liu criterion; :AMD and :MDQ), reverse Cuthill-McKee (:RCM), or
//      the natural order;
//   2. left-looking sparse LU of A(:, q) with threshold partial pivoting (Gilbert-Peierls:
//      depth-first reach in the graph of L, then a sparse triangular solve per column);
//      threshold 1.0 as the reference passes to csrluFactorHost (:148);
//   3. the structural L + U pattern of A_hat = A(P, q) in CSR, and the map from A's entries
//      into it.
// Device side: the numeric factorization is the same level-scheduled cooperative kernel as
// ILU(0), run on the L + U pattern (no fill is dropped, so it is the exact LU with the fixed
// pivot order), and the solve is one cooperative launch of both triangular sweeps with the
// row permutation P fused into the layout conversion on the way in and Q on the way out.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <queue>
#include <set>
#include <vector>

#include "bpf_internal.cuh"
#include "ordering.cuh"
#include "prec.cuh"

namespace bpf {

// ------------------------------------------------------------------------------------
// left-looking sparse LU with threshold partial pivoting (Gilbert-Peierls)
// ------------------------------------------------------------------------------------
struct HostLU {
    std::vector<int> Lp, Li;   // L columns (strict lower), row ids in ORIGINAL numbering
    std::vector<double> Lx;
    std::vector<int> Up, Ui;   // U columns incl. diagonal, row ids in pivot-step numbering
    std::vector<double> Ux;
    std::vector<int> pinv;     // original row -> pivot step
    std::vector<int> P;        // pivot step -> original row
};

static int sparse_lu(int n, const std::vector<int> &cp, const std::vector<int> &ri,
                     const std::vector<double> &cv, const std::vector<int> &q, double thresh,
                     double tol, HostLU &lu, int *bad_col) {
    lu.Lp.assign(n + 1, 0);
    lu.Up.assign(n + 1, 0);
    lu.Li.clear(); lu.Lx.clear(); lu.Ui.clear(); lu.Ux.clear();
    lu.pinv.assign(n, -1);
    lu.P.assign(n, -1);
    std::vector<double> x(n, 0.0);
    std::vector<int> mark(n, -1), topo, stack_node, stack_pos;
    topo.reserve(n);
    for (int k = 0; k < n; k++) {
        const int col = q[k];
        topo.clear();
        // depth-first reach of A(:, col) in the graph of L (post-order in topo)
        for (int t = cp[col]; t < cp[col + 1]; t++) {
            int r0 = ri[t];
            if (mark[r0] == k) continue;
            stack_node.assign(1, r0);
            stack_pos.assign(1, 0);
            mark[r0] = k;
            while (!stack_node.empty()) {
                int r = stack_node.back();
                int j = lu.pinv[r];
                int &pos = stack_pos.back();
                bool pushed = false;
                if (j >= 0) {
                    for (int e = lu.Lp[j] + pos; e < lu.Lp[j + 1]; e++) {
                        int i = lu.Li[e];
                        pos++;
                        if (mark[i] != k) {
                            mark[i] = k;
                            stack_node.push_back(i);
                            stack_pos.push_back(0);
                            pushed = true;
                            break;
                        }
                    }
                }
                if (!pushed) {
                    topo.push_back(r);
                    stack_node.pop_back();
                    stack_pos.pop_back();
                }
            }
        }
        for (int t = cp[col]; t < cp[col + 1]; t++) x[ri[t]] = cv[t];
        // sparse triangular solve in topological order (reverse post-order)
        for (int t = (int)topo.size() - 1; t >= 0; t--) {
            int r = topo[t];
            int j = lu.pinv[r];
            if (j < 0) continue;
            double xj = x[r];
            for (int e = lu.Lp[j]; e < lu.Lp[j + 1]; e++) x[lu.Li[e]] -= lu.Lx[e] * xj;
        }
        // pivot among not-yet-pivoted rows; prefer the diagonal row q[k] within the threshold
        int piv = -1;
        double amax = -1.0;
        for (int r : topo)
            if (lu.pinv[r] < 0 && std::fabs(x[r]) > amax) {
                amax = std::fabs(x[r]);
                piv = r;
            }
        if (piv >= 0 && lu.pinv[col] < 0 && mark[col] == k && std::fabs(x[col]) >= thresh * amax) piv = col;
        if (piv < 0 || !(std::fabs(x[piv]) > tol)) {
            *bad_col = k;
            return -1;
        }
        const double pv = x[piv];
        // U(:, k): pivoted rows in the reach, then the diagonal
        for (int r : topo) {
            int j = lu.pinv[r];
            if (j >= 0) {
                lu.Ui.push_back(j);
                lu.Ux.push_back(x[r]);
            }
        }
        lu.Ui.push_back(k);
        lu.Ux.push_back(pv);
        lu.Up[k + 1] = (int)lu.Ui.size();
        for (int r : topo) {
            if (lu.pinv[r] < 0 && r != piv) {
                lu.Li.push_back(r);
                lu.Lx.push_back(x[r] / pv);
            }
        }
        lu.Lp[k + 1] = (int)lu.Li.size();
        lu.pinv[piv] = k;
        lu.P[k] = piv;
        for (int r : topo) x[r] = 0.0;
    }
    return 0;
}

// ------------------------------------------------------------------------------------
// device helpers: permuted layout conversions and value scatter
// ------------------------------------------------------------------------------------
// dst[i][c] = src[c*ld + perm[i]]  (column-major -> row-major, gathering rows)
// X (column-major, ld ldx) += R (n x p, ld n).
__global__ void cm_add_kernel(int n, int p, const double *__restrict__ R, double *__restrict__ X, int ldx) {
    const size_t len = (size_t)n * p;
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < len; idx += (size_t)gridDim.x * blockDim.x) {
        const size_t c = idx / n, r = idx - c * n;
        X[c * ldx + r] += R[idx];
    }
}

__global__ void cm_to_rm_perm_kernel(int n, int p, const double *__restrict__ src, int ld,
                                     const int *__restrict__ perm, double *__restrict__ dst) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * p;
         e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / p), c = (int)(e % p);
        dst[e] = src[(size_t)c * ld + perm[i]];
    }
}

// dst[c*ld + perm[j]] = src[j][c]  (row-major -> column-major, scattering rows)
__global__ void rm_to_cm_perm_kernel(int n, int p, const double *__restrict__ src,
                                     const int *__restrict__ perm, double *__restrict__ dst, int ld) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * p;
         e += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / p), c = (int)(e % p);
        dst[(size_t)c * ld + perm[j]] = src[e];
    }
}

__global__ void scatter_vals_kernel(int nnzA, const double *__restrict__ vals,
                                    const int *__restrict__ amap, double *__restrict__ fv) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnzA; e += gridDim.x * blockDim.x)
        fv[amap[e]] = vals[e];
}

}  // namespace bpf

// The RF object (CusolverRfLU / CusolverRfLUBatch).
struct bpf_rf {
    bpf_ctx *ctx = nullptr;
    int n = 0, nnzA = 0, batch = 1, fast_mode = 1, ordering = 0;
    int nnzL = 0, nnzU = 0;
    std::vector<int> P, Q;            // host permutations (0-based)
    int *Pd = nullptr, *Qd = nullptr; // device copies
    int *amap = nullptr;              // A entry -> L+U position
    bpf_prec *lu = nullptr;           // pattern, schedules and factor of the (uniform) matrix
    bool uniform = true;              // all batch replicas hold the same values
    // per-replica factor values (batch mode after rf_batch_refactor with distinct columns)
    std::vector<double *> rep_lval, rep_uval, rep_dinv;
};

namespace bpf {

static bpf_status rf_factor_values(bpf_rf *rf, const double *vals) {
    bpf_ctx *ctx = rf->ctx;
    bpf_prec *P = rf->lu;
    BPF_CUDA(ctx, cudaMemsetAsync(P->fv, 0, sizeof(double) * P->nnz, ctx->stream));
    if (rf->nnzA > 0) {
        int blocks = std::min(ceil_div(rf->nnzA, 256), ctx->num_sms * 8);
        scatter_vals_kernel<<<blocks, 256, 0, ctx->stream>>>(rf->nnzA, vals, rf->amap, P->fv);
        BPF_LAUNCHED(ctx);
    }
    BPF_TRY(factor_numeric(ctx, P));
    BPF_TRY(tri_scatter(ctx, P->lower, P->fv));
    BPF_TRY(tri_scatter(ctx, P->upper, P->fv));
    return BPF_SUCCESS;
}

static void rf_free_replicas(bpf_rf *rf) {
    for (double *p : rf->rep_lval) cudaFree(p);
    for (double *p : rf->rep_uval) cudaFree(p);
    for (double *p : rf->rep_dinv) cudaFree(p);
    rf->rep_lval.clear();
    rf->rep_uval.clear();
    rf->rep_dinv.clear();
}

}  // namespace bpf

using namespace bpf;

extern "C" {

bpf_status bpf_rf_analyze(bpf_ctx *ctx, const bpf_csr_desc *A, int ordering, double tol,
                          int fast_mode, int batch, bpf_rf **out) {
    if (!ctx || !out) return BPF_ERR_INVALID_VALUE;
    *out = nullptr;
    if (!A) return set_error(ctx, BPF_ERR_INVALID_VALUE, "null matrix");
    if (A->dtype != BPF_F64) return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "FP64 matrices only");
    if (batch < 1) return set_error(ctx, BPF_ERR_INVALID_VALUE, "batch must be >= 1");
    if (ordering == BPF_ORDER_METIS)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED,
                         "ordering :METIS needs a METIS library, which this build does not link");
    if (ordering < 0 || ordering > BPF_ORDER_NATURAL)
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "unknown ordering %d", ordering);
    std::vector<int> rp, ci;
    BPF_TRY(csr_pattern_to_host(ctx, A, rp, ci, false, nullptr));
    const int n = A->n, nnz = A->nnz;
    std::vector<double> av(nnz);
    if (nnz > 0)
        BPF_CUDA(ctx, cudaMemcpy(av.data(), A->vals, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
    // 1. ordering
    std::vector<int> q;
    if (ordering == BPF_ORDER_AMD || ordering == BPF_ORDER_MDQ) q = order_min_degree(n, rp, ci);
    else if (ordering == BPF_ORDER_RCM) q = order_rcm(n, rp, ci);
    else {
        q.resize(n);
        for (int i = 0; i < n; i++) q[i] = i;
    }
    // 2. CSC of A and the pivoted LU of A(:, q)
    std::vector<int> cp(n + 1, 0), rix(nnz), cpos(nnz);
    std::vector<double> cv(nnz);
    for (int k = 0; k < nnz; k++) cp[ci[k] + 1]++;
    for (int j = 0; j < n; j++) cp[j + 1] += cp[j];
    {
        std::vector<int> fill(cp.begin(), cp.end() - 1);
        for (int i = 0; i < n; i++)
            for (int k = rp[i]; k < rp[i + 1]; k++) {
                int d = fill[ci[k]]++;
                rix[d] = i;
                cv[d] = av[k];
                cpos[d] = k;
            }
    }
    HostLU lu;
    int bad = -1;
    if (sparse_lu(n, cp, rix, cv, q, 1.0, tol, lu, &bad) != 0)
        return set_error(ctx, BPF_ERR_SINGULAR, "rf_analyze: zero pivot (|pivot| <= tol=%g) at column %d", tol, bad);
    // 3. L + U pattern of A_hat = A(P, q) in CSR (pivot-step numbering)
    std::vector<int> qinv(n);
    for (int j = 0; j < n; j++) qinv[q[j]] = j;
    std::vector<std::vector<int>> rows(n);
    for (int j = 0; j < n; j++)
        for (int e = lu.Lp[j]; e < lu.Lp[j + 1]; e++) rows[lu.pinv[lu.Li[e]]].push_back(j);
    for (int k = 0; k < n; k++)
        for (int e = lu.Up[k]; e < lu.Up[k + 1]; e++) rows[lu.Ui[e]].push_back(k);
    std::vector<int> Frp(n + 1, 0), Fci, Fdiag(n, -1);
    for (int i = 0; i < n; i++) {
        std::sort(rows[i].begin(), rows[i].end());
        Frp[i + 1] = Frp[i] + (int)rows[i].size();
    }
    Fci.reserve(Frp[n]);
    for (int i = 0; i < n; i++) {
        for (int c : rows[i]) {
            if (c == i) Fdiag[i] = (int)Fci.size();
            Fci.push_back(c);
        }
        std::vector<int>().swap(rows[i]);
    }
    // map A entries into the pattern
    std::vector<int> amap(nnz);
    for (int i = 0; i < n; i++) {
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            const int r = lu.pinv[i], c = qinv[ci[k]];
            auto b = Fci.begin() + Frp[r], e = Fci.begin() + Frp[r + 1];
            auto it = std::lower_bound(b, e, c);
            if (it == e || *it != c) return set_error(ctx, BPF_ERR_INVALID_VALUE, "rf_analyze: pattern map failed");
            amap[k] = (int)(it - Fci.begin());
        }
    }
    bpf_rf *rf = new bpf_rf();
    rf->ctx = ctx;
    rf->n = n;
    rf->nnzA = nnz;
    rf->batch = batch;
    rf->fast_mode = fast_mode;
    rf->ordering = ordering;
    rf->nnzL = (int)lu.Li.size();
    rf->nnzU = (int)lu.Ui.size();
    rf->P = lu.P;
    rf->Q = q;
    auto fail = [&](bpf_status s) {
        cudaStreamSynchronize(ctx->stream);
        bpf_rf_destroy(rf);
        return s;
    };
    bpf_status s = prec_setup(ctx, PREC_LU, n, Frp, Fci, Fdiag, &rf->lu);
    if (s != BPF_SUCCESS) return fail(s);
    rf->lu->fdtype = BPF_F64;
    cudaError_t e = cudaMalloc((void **)&rf->Pd, sizeof(int) * std::max(n, 1));
    if (e == cudaSuccess) e = cudaMalloc((void **)&rf->Qd, sizeof(int) * std::max(n, 1));
    if (e == cudaSuccess) e = cudaMalloc((void **)&rf->amap, sizeof(int) * std::max(nnz, 1));
    if (e == cudaSuccess && n > 0) e = cudaMemcpy(rf->Pd, rf->P.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n > 0) e = cudaMemcpy(rf->Qd, rf->Q.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nnz > 0) e = cudaMemcpy(rf->amap, amap.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(cuda_error(ctx, e, "rf setup", __FILE__, __LINE__));
    // device refactor of A's own values (the reference runs Analyze + Refactor here, :293-295)
    if ((s = rf_factor_values(rf, (const double *)A->vals)) != BPF_SUCCESS) return fail(s);
    if ((s = check_dev_status(ctx, "rf_analyze")) != BPF_SUCCESS) return fail(s);
    *out = rf;
    return BPF_SUCCESS;
}

bpf_status bpf_rf_refactor(bpf_rf *rf, const double *vals) {
    if (!rf) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = rf->ctx;
    if (rf->nnzA > 0 && !vals) return set_error(ctx, BPF_ERR_INVALID_VALUE, "null values");
    rf_free_replicas(rf);
    rf->uniform = true;
    BPF_TRY(rf_factor_values(rf, vals));
    return check_dev_status(ctx, "rf_refactor");
}

bpf_status bpf_rf_refactor_batch(bpf_rf *rf, const double *vals, int ld) {
    if (!rf) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = rf->ctx;
    if (rf->nnzA > 0 && !vals) return set_error(ctx, BPF_ERR_INVALID_VALUE, "null values");
    if (ld < rf->nnzA) return set_error(ctx, BPF_ERR_DIMENSION, "rf_refactor_batch: ld < nnz");
    if (rf->batch == 1) return bpf_rf_refactor(rf, vals);
    rf_free_replicas(rf);
    rf->uniform = false;
    bpf_prec *P = rf->lu;
    const int n = rf->n;
    for (int r = 0; r < rf->batch; r++) {
        BPF_TRY(rf_factor_values(rf, vals + (size_t)r * ld));
        double *lv = nullptr, *uv = nullptr, *dv = nullptr;
        BPF_CUDA(ctx, cudaMalloc((void **)&lv, sizeof(double) * std::max(P->lower.nnz, 1)));
        rf->rep_lval.push_back(lv);
        BPF_CUDA(ctx, cudaMalloc((void **)&uv, sizeof(double) * std::max(P->upper.nnz, 1)));
        rf->rep_uval.push_back(uv);
        BPF_CUDA(ctx, cudaMalloc((void **)&dv, sizeof(double) * std::max(n, 1)));
        rf->rep_dinv.push_back(dv);
        if (P->lower.nnz)
            BPF_CUDA(ctx, cudaMemcpyAsync(lv, P->lower.val, sizeof(double) * P->lower.nnz,
                                          cudaMemcpyDeviceToDevice, ctx->stream));
        if (P->upper.nnz)
            BPF_CUDA(ctx, cudaMemcpyAsync(uv, P->upper.val, sizeof(double) * P->upper.nnz,
                                          cudaMemcpyDeviceToDevice, ctx->stream));
        BPF_CUDA(ctx, cudaMemcpyAsync(dv, P->upper.dinv, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
    }
    return check_dev_status(ctx, "rf_refactor_batch");
}

bpf_status bpf_rf_solve(bpf_rf *rf, int nrhs, double *X, int ldx) {
    if (!rf) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = rf->ctx;
    const int n = rf->n;
    if (nrhs < 0 || (nrhs > 0 && n > 0 && !X)) return set_error(ctx, BPF_ERR_INVALID_VALUE, "rf_solve: invalid argument");
    if (ldx < std::max(1, n)) return set_error(ctx, BPF_ERR_DIMENSION, "rf_solve: ldx < n");
    if (rf->batch > 1 && nrhs != rf->batch)
        return set_error(ctx, BPF_ERR_DIMENSION, "batch mode solves exactly batchsize=%d columns", rf->batch);
    if (n == 0 || nrhs == 0) return BPF_SUCCESS;
    const int chunk = 256;
    bpf_status s;
    double *buf = (double *)ws_get(ctx, WS_A, sizeof(double) * (size_t)n * std::min(nrhs, chunk), &s);
    if (!buf) return s;
    auto conv_in = [&](int c0, int pc) -> bpf_status {
        size_t len = (size_t)n * pc;
        int blocks = std::max(1, std::min(ceil_div((long long)len, 256), ctx->num_sms * 8));
        cm_to_rm_perm_kernel<<<blocks, 256, 0, ctx->stream>>>(n, pc, X + (size_t)c0 * ldx, ldx, rf->Pd, buf);
        BPF_LAUNCHED(ctx);
        return BPF_SUCCESS;
    };
    auto conv_out = [&](int c0, int pc) -> bpf_status {
        size_t len = (size_t)n * pc;
        int blocks = std::max(1, std::min(ceil_div((long long)len, 256), ctx->num_sms * 8));
        rm_to_cm_perm_kernel<<<blocks, 256, 0, ctx->stream>>>(n, pc, buf, rf->Qd, X + (size_t)c0 * ldx, ldx);
        BPF_LAUNCHED(ctx);
        return BPF_SUCCESS;
    };
    if (rf->uniform) {
        for (int c0 = 0; c0 < nrhs; c0 += chunk) {
            int pc = std::min(chunk, nrhs - c0);
            BPF_TRY(conv_in(c0, pc));
            if (rf->lu->ps_nlev[0] + rf->lu->ps_nlev[1] > 0)
                BPF_TRY(lu_solve_push_rowmajor(ctx, rf->lu, pc, buf));
            else
                BPF_TRY(prec_apply_rowmajor(ctx, rf->lu, pc, buf, buf));
            BPF_TRY(conv_out(c0, pc));
        }
        return BPF_SUCCESS;
    }
    // distinct replicas: column r with replica r's factors
    bpf_prec *P = rf->lu;
    double *lv0 = P->lower.val, *uv0 = P->upper.val, *dv0 = P->upper.dinv;
    for (int r = 0; r < nrhs; r++) {
        P->lower.val = rf->rep_lval[r];
        P->upper.val = rf->rep_uval[r];
        P->upper.dinv = rf->rep_dinv[r];
        bpf_status st = conv_in(r, 1);
        if (st == BPF_SUCCESS) st = prec_apply_rowmajor(ctx, P, 1, buf, buf);
        if (st == BPF_SUCCESS) st = conv_out(r, 1);
        P->lower.val = lv0;
        P->upper.val = uv0;
        P->upper.dinv = dv0;
        if (st != BPF_SUCCESS) return st;
    }
    return BPF_SUCCESS;
}

bpf_status bpf_rf_solve_refined(bpf_rf *rf, const bpf_csr_desc *A, int nrhs, const double *B, int ldb,
                                double *X, int ldx, int steps) {
    if (!rf) return BPF_ERR_INVALID_VALUE;
    bpf_ctx *ctx = rf->ctx;
    const int n = rf->n;
    if (!A || nrhs < 0 || steps < 0 || (nrhs > 0 && n > 0 && (!B || !X)))
        return set_error(ctx, BPF_ERR_INVALID_VALUE, "rf_solve_refined: invalid argument");
    if (A->n != n || A->nnz != rf->nnzA)
        return set_error(ctx, BPF_ERR_DIMENSION, "rf_solve_refined: A is not the analysed matrix");
    if (ldb < std::max(1, n) || ldx < std::max(1, n))
        return set_error(ctx, BPF_ERR_DIMENSION, "rf_solve_refined: leading dimension < n");
    if (!rf->uniform)
        return set_error(ctx, BPF_ERR_NOT_SUPPORTED, "rf_solve_refined: replicas with distinct values");
    if (rf->batch > 1 && nrhs != rf->batch)
        return set_error(ctx, BPF_ERR_DIMENSION, "batch mode solves exactly batchsize=%d columns", rf->batch);
    if (n == 0 || nrhs == 0) return BPF_SUCCESS;
    BPF_CUDA(ctx, cudaMemcpy2DAsync(X, sizeof(double) * ldx, B, sizeof(double) * ldb, sizeof(double) * n, nrhs,
                                    cudaMemcpyDeviceToDevice, ctx->stream));
    BPF_TRY(bpf_rf_solve(rf, nrhs, X, ldx));
    if (steps == 0) return BPF_SUCCESS;
    bpf_status st;
    double *R = (double *)ws_get(ctx, WS_C, sizeof(double) * (size_t)n * nrhs, &st);
    if (!R) return st;
    for (int k = 0; k < steps; k++) {
        // R = B - A X, then X += LU \ R
        BPF_CUDA(ctx, cudaMemcpy2DAsync(R, sizeof(double) * n, B, sizeof(double) * ldb, sizeof(double) * n, nrhs,
                                        cudaMemcpyDeviceToDevice, ctx->stream));
        BPF_TRY(bpf_spmm(ctx, A, nrhs, -1.0, X, ldx, 1.0, R, n));
        BPF_TRY(bpf_rf_solve(rf, nrhs, R, n));
        const size_t len = (size_t)n * nrhs;
        const int blocks = std::max(1, std::min(ceil_div((long long)len, 256), ctx->num_sms * 8));
        cm_add_kernel<<<blocks, 256, 0, ctx->stream>>>(n, nrhs, R, X, ldx);
        BPF_LAUNCHED(ctx);
    }
    return BPF_SUCCESS;
}

bpf_status bpf_rf_info(const bpf_rf *rf, int *nnzL, int *nnzU, int *P, int *Q) {
    if (!rf) return BPF_ERR_INVALID_VALUE;
    if (nnzL) *nnzL = rf->nnzL;
    if (nnzU) *nnzU = rf->nnzU;
    if (P && rf->n) std::memcpy(P, rf->P.data(), sizeof(int) * rf->n);
    if (Q && rf->n) std::memcpy(Q, rf->Q.data(), sizeof(int) * rf->n);
    return BPF_SUCCESS;
}

bpf_status bpf_rf_destroy(bpf_rf *rf) {
    if (!rf) return BPF_SUCCESS;
    if (rf->ctx) cudaStreamSynchronize(rf->ctx->stream);
    rf_free_replicas(rf);
    if (rf->lu) bpf_prec_destroy(rf->lu);
    cudaFree(rf->Pd);
    cudaFree(rf->Qd);
    cudaFree(rf->amap);
    delete rf;
    return BPF_SUCCESS;
}

}  // extern "C"
